"""In-tree build of the native library (libfgpe.so, sm_100a) and the drop-in
driver executable (cgpe.x)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(verbose=False):
    env = dict(os.environ)
    # use the toolchain on PATH (nvcc drives the host compiler itself)
    env.pop("CC", None)
    env.pop("CXX", None)
    # the translation units compile in parallel (the largest takes minutes)
    cmd = ["make", "-j", str(max(2, min(8, os.cpu_count() or 2))), "-C", os.path.join(HERE, "csrc")]
    if not verbose:
        cmd.insert(1, "-s")
    subprocess.run(cmd, check=True, env=env)
    return os.path.join(HERE, "libfgpe.so")


if __name__ == "__main__":
    print(build(verbose=True))
