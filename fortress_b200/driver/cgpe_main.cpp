// cgpe_main.cpp -- drop-in replacement for FORTRESS's ./cgpe.x.
//
// Built once per dimension (FGPE_DIMENSION = 1, 2 or 3, like the reference's
// Makefile DIMENSION switch).  Reads ./INPUT/input{1,2,3}D.dat (and, in real
// time, ./INPUT/initial_sol_spin{1,2}.dat), writes ./OUTPUT/file1..3, the
// solution and transient-solution files and convergence.dat with the
// reference's formats, and ./err_msg.dat.  Program flow restates PROGRAM
// CGPE1D/2D/3D (cgpe1d.f90:212-563, cgpe2d.f90:212-579, cgpe3d.f90:217-617);
// the propagation runs on the GPU through the C ABI of include/fgpe.h.
//
// Extension (not an input record): FGPE_PRECISION=fp32 in the environment
// selects the FP32-bulk path.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <sys/time.h>

#include <algorithm>
#include <complex>
#include <string>
#include <vector>

#include "../../include/fgpe.h"

#ifndef FGPE_DIMENSION
#define FGPE_DIMENSION 3
#endif

typedef std::complex<double> cd;

static const double PI = 3.14159265358979323846264338327950288;
static const double AMU = 1.66e-27, HBAR = 1.054560653e-34, AU = 0.529177208e-10, EPS = 1.0e-40;

// ------------------------------------------------------ Fortran editing
// Fw.d (asterisks when the value does not fit).
static std::string fF(double x, int w, int d) {
    char b[128];
    snprintf(b, sizeof b, "%.*f", d, x);
    std::string s(b);
    if ((int)s.size() > w && s.compare(0, 2, "0.") == 0) s = s.substr(1);       // drop optional leading 0
    if ((int)s.size() > w && s.compare(0, 3, "-0.") == 0) s = "-" + s.substr(2);
    if ((int)s.size() > w) return std::string(w, '*');
    return std::string(w - s.size(), ' ') + s;
}
static std::string fI(long long v, int w) {
    char b[64];
    snprintf(b, sizeof b, "%lld", v);
    std::string s(b);
    if ((int)s.size() > w) return std::string(w, '*');
    return std::string(w - s.size(), ' ') + s;
}
// Ew.d: 0.ddddE+ee
static std::string fE(double x, int w, int d) {
    char b[128];
    if (x == 0.0) {
        snprintf(b, sizeof b, "0.%0*dE+00", d, 0);
    } else {
        int e = (int)floor(log10(fabs(x))) + 1;
        double m = x / pow(10.0, e);
        char mb[64];
        snprintf(mb, sizeof mb, "%.*f", d, fabs(m));
        if (mb[0] == '1') { e += 1; m /= 10.0; snprintf(mb, sizeof mb, "%.*f", d, fabs(m)); }
        snprintf(b, sizeof b, "%s%sE%c%02d", x < 0 ? "-" : "", mb, e < 0 ? '-' : '+', abs(e));
    }
    std::string s(b);
    if ((int)s.size() > w) return std::string(w, '*');
    return std::string(w - s.size(), ' ') + s;
}
// ESw.d: d.ddE+ee
static std::string fES(double x, int w, int d) {
    char b[128];
    snprintf(b, sizeof b, "%.*E", d, x);
    std::string s(b);
    if ((int)s.size() > w) return std::string(w, '*');
    return std::string(w - s.size(), ' ') + s;
}
// List-directed REAL(8) item as the reference output shows it: 24 columns,
// G editing with 15 significant digits (F form plus 5 blanks for
// 0.1 <= |x| < 1e15, otherwise d.ddddE-eee).
static std::string fList(double x) {
    const double a = fabs(x);
    char b[128];
    if (a >= 0.1 && a < 1e15) {
        int k = (int)floor(log10(a)) + 1;
        snprintf(b, sizeof b, "%.*f", 15 - k, x);
        // rounding can carry into a new digit (e.g. 9.99.. -> 10.0..)
        if ((int)strlen(b) > 17 + (x < 0)) snprintf(b, sizeof b, "%.*f", 15 - k - 1, x);
        std::string s(b);
        return std::string(19 - (int)s.size() > 0 ? 19 - s.size() : 0, ' ') + s + "     ";
    }
    if (x == 0.0) return std::string("  0.000000000000000E+000");
    int e = (int)floor(log10(a));
    double m = x / pow(10.0, e);
    snprintf(b, sizeof b, "%.15f", fabs(m));
    if (b[0] == '1' && b[1] == '0') { e += 1; m /= 10.0; snprintf(b, sizeof b, "%.15f", fabs(m)); }
    char o[128];
    snprintf(o, sizeof o, "%s%sE%c%03d", x < 0 ? "-" : "", b, e < 0 ? '-' : '+', abs(e));
    std::string s(o);
    return std::string(24 - (int)s.size() > 0 ? 24 - s.size() : 0, ' ') + s;
}

// --------------------------------------------------- list-directed input
struct Reader {
    FILE* f;
    bool eof = false;
    // tokens of the next record(s) until n values are read (rest of the last
    // record is discarded, like a Fortran list-directed READ)
    bool read(std::vector<double>& out, size_t n) {
        out.clear();
        char line[4096];
        while (out.size() < n) {
            if (!fgets(line, sizeof line, f)) { eof = true; return false; }
            char* p = line;
            while (*p && out.size() < n) {
                while (*p == ' ' || *p == '\t' || *p == ',' || *p == '\n' || *p == '\r') ++p;
                if (!*p || *p == '/') break;
                char tok[256];
                int k = 0;
                while (*p && *p != ' ' && *p != '\t' && *p != ',' && *p != '\n' && *p != '\r' && k < 255) tok[k++] = *p++;
                tok[k] = 0;
                for (int i = 0; i < k; ++i) if (tok[i] == 'D' || tok[i] == 'd') tok[i] = 'E';
                char* star = strchr(tok, '*');
                int rep = 1;
                const char* val = tok;
                if (star) { *star = 0; rep = atoi(tok); val = star + 1; }
                char* end = nullptr;
                double v = strtod(val, &end);
                if (end == val) { out.clear(); return false; }   // not a number
                for (int r = 0; r < rep && out.size() < n; ++r) out.push_back(v);
            }
        }
        return true;
    }
    bool skip() {
        char line[4096];
        if (!fgets(line, sizeof line, f)) { eof = true; return false; }
        return true;
    }
};

static void date_line(FILE* f, const char* what) {
    time_t t = time(nullptr);
    struct tm lt;
    localtime_r(&t, &lt);
    // (I2,'/',I2,'/',I4,',',I3,':',I2,':',I2)
    fprintf(f, "%s on DAY/MONTH/YEAR, HOURS:MINUTES:SECONDS = %s/%s/%s,%s:%s:%s\n", what, fI(lt.tm_mday, 2).c_str(),
            fI(lt.tm_mon + 1, 2).c_str(), fI(lt.tm_year + 1900, 4).c_str(), fI(lt.tm_hour, 3).c_str(),
            fI(lt.tm_min, 2).c_str(), fI(lt.tm_sec, 2).c_str());
}

static double wall() {
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return tv.tv_sec + 1e-6 * tv.tv_usec;
}

static FILE* g_err = nullptr;

static void stop_with(const std::string& msg) {
    fprintf(g_err, " %s\n", msg.c_str());
    printf(" %s\n", msg.c_str());
    fclose(g_err);
    exit(0);  // Fortran STOP
}

static void check(int rc, fgpe_t* h) {
    if (rc == FGPE_OK) return;
    std::string m = fgpe_last_error(h);
    if (rc == FGPE_E_NEWTON)
        stop_with("Newton-Raphason subroutine could not calculate the roots within   1.000000000000000E-006  tolerance");
    stop_with("fgpe error: " + m);
}

int main() {
    const int D = FGPE_DIMENSION;
    const double t_start = wall();
    const std::string dtag = std::to_string(D) + "D";
    FILE* ferr = fopen("err_msg.dat", "w");
    g_err = ferr;
    const std::string in_path = "./INPUT/input" + dtag + ".dat";
    FILE* fin = fopen(in_path.c_str(), "r");
    if (!fin) stop_with("'input" + dtag + ".dat' does not exist.");
    date_line(stdout, "Started");  // console echo; file1 gets its own line below

    // ---------------------------------------------- input records
    Reader rd{fin};
    std::vector<double> v;
    auto need = [&](size_t n) { if (!rd.read(v, n)) stop_with("error reading " + in_path); };
    need(1); const int SPIN = (int)v[0];
    need(1); const long long NITER = (long long)v[0];
    need(2); const long long STP = (long long)v[0], NSTP = (long long)v[1];
    need(1); const int THREADS = (int)v[0];
    need(D); int N[3] = {1, 1, 1}; for (int a = 0; a < D; ++a) N[a] = (int)v[a];
    need(D + 1); double DX[3] = {1, 1, 1}; for (int a = 0; a < D; ++a) DX[a] = v[a]; const double DT = v[D];
    need(1); const double MASS = v[0];
    need(SPIN == 1 ? 2 : 3); const double A0 = v[0], A2 = v[1], A4 = SPIN == 2 ? v[2] : 0.0;
    need(1); const long long NATOMS = (long long)v[0];
    need(3); const double NUX = v[0], NUY = v[1], NUZ = v[2];
    need(1); const double TOL = v[0];
    need(1); const int SWITCH_IM = (int)v[0];
    need(D); double G[3] = {0, 0, 0}; for (int a = 0; a < D; ++a) G[a] = v[a];
    int SWITCH_SOC = 0;
    for (int a = 0; a < D; ++a) if (fabs(G[a]) > EPS) SWITCH_SOC = 1;
    int OPTION_FPC = 4;
    double MAG = 0.0;
    if (SWITCH_SOC == 0) { need(1); OPTION_FPC = (int)v[0]; } else rd.skip();
    if (SWITCH_IM == 1 && SWITCH_SOC == 0) { need(1); MAG = v[0]; } else rd.skip();
    fclose(fin);
    if (SPIN != 1 && SPIN != 2) stop_with("SPIN must be 1 or 2");
    const int MS = 2 * SPIN + 1;
    const double ALPHAX = NUX / NUX, ALPHAY = NUY / NUX, ALPHAZ = NUZ / NUX;
    const double AL[3] = {ALPHAX, ALPHAY, ALPHAZ};
    const char* sid = SPIN == 1 ? "1" : "2";
    printf(" MAXIMUM_THREAD_NUMBER_SET = %12d\n", THREADS);

    // ---------------------------------------------- output files
    const std::string im = SWITCH_IM == 1 ? "im" : "re";
    FILE* f1 = fopen(("./OUTPUT/file1_" + im + "_spin" + sid + ".dat").c_str(), "w");
    FILE* f2 = fopen(("./OUTPUT/file2_" + im + "_spin" + sid + ".dat").c_str(), "w");
    FILE* f3 = fopen(("./OUTPUT/file3_" + im + "_spin" + sid + ".dat").c_str(), "w");
    FILE* f8 = fopen(("./OUTPUT/solution_file_" + im + "_spin" + sid + ".dat").c_str(), "w");
    FILE* f9 = SWITCH_IM == 1 ? fopen("./OUTPUT/convergence.dat", "w") : nullptr;
    if (!f1 || !f2 || !f3 || !f8 || (SWITCH_IM == 1 && !f9)) stop_with("cannot open files in ./OUTPUT");
    FILE* finit = nullptr;
    if (SWITCH_IM != 1) finit = fopen((std::string("./INPUT/initial_sol_spin") + sid + ".dat").c_str(), "r");
    date_line(f1, "Started");

    // ---------------------------------------------- AOSC, TAU
    const double OMEGAM = 2.0 * PI * NUX;
    const double AOSC = sqrt(HBAR / (MASS * AMU * OMEGAM));
    const double geo = D == 1 ? sqrt(ALPHAY * ALPHAZ) / (2.0 * PI) : D == 2 ? sqrt(ALPHAZ / (2.0 * PI)) : 1.0;
    double TAU[3] = {0, 0, 0};
    if (SPIN == 1) {
        const double na = (double)(float)NATOMS;   // REAL(NATOMS)
        TAU[0] = 2.0 * geo * (4.0 * PI * na * (A0 * AU + 2.0 * A2 * AU) / (3.0 * AOSC));
        TAU[1] = 2.0 * geo * (4.0 * PI * na * (A2 * AU - A0 * AU) / (3.0 * AOSC));
    } else {
        const double nd = (double)NATOMS;
        TAU[0] = 2.0 * (geo * 4.0 * PI * nd * (4.0 * A2 * AU + 3.0 * A4 * AU) / (7.0 * AOSC));
        TAU[1] = 2.0 * (geo * 4.0 * PI * nd * (A4 * AU - A2 * AU) / (7.0 * AOSC));
        TAU[2] = 2.0 * (geo * 4.0 * PI * nd * (7.0 * A0 * AU - 10.0 * A2 * AU + 3.0 * A4 * AU) / (7.0 * AOSC));
    }

    // ---------------------------------------------- file1 header
    fprintf(f1, " \n");
    fprintf(f1, " OPENMP_THREADS = %s, FFTW_THREADS = %s\n", fI(THREADS, 3).c_str(), fI(THREADS, 3).c_str());
    if (D == 1)
        fprintf(f1, " SWITCH_IM = %s, OPTION_FPC = %s, SWITCH_SOC = %s, GAMMAX = %s, TOL = %s\n", fI(SWITCH_IM, 2).c_str(),
                fI(OPTION_FPC, 2).c_str(), fI(SWITCH_SOC, 2).c_str(), fF(G[0], 6, 2).c_str(), fES(TOL, 9, 2).c_str());
    else if (D == 2)
        fprintf(f1, " SWITCH_IM = %s, OPTION_FPC = %s, SWITCH_SOC = %s, GAMMAX = %s, GAMMAY = %s, TOL = %s\n",
                fI(SWITCH_IM, 2).c_str(), fI(OPTION_FPC, 2).c_str(), fI(SWITCH_SOC, 2).c_str(), fF(G[0], 6, 2).c_str(),
                fF(G[1], 6, 2).c_str(), fES(TOL, 9, 2).c_str());
    else
        fprintf(f1, " SWITCH_IM = %s, OPTION_FPC = %s, SWITCH_SOC = %s, GAMMAX = %s, GAMMAY = %s, GAMMAZ = %s, TOL = %s\n",
                fI(SWITCH_IM, 2).c_str(), fI(OPTION_FPC, 2).c_str(), fI(SWITCH_SOC, 2).c_str(), fF(G[0], 6, 2).c_str(),
                fF(G[1], 6, 2).c_str(), fF(G[2], 6, 2).c_str(), fES(TOL, 9, 2).c_str());
    fprintf(f1, " Anisotropy ALPHAX =%s%s, ALPHAY = %s, ALPHAZ = %s\n", D == 1 ? " " : "", fF(ALPHAX, 12, 6).c_str(),
            fF(ALPHAY, 12, 6).c_str(), fF(ALPHAZ, 12, 6).c_str());
    fprintf(f1, " \n");
    if (D == 1) fprintf(f1, " No. of space steps NX = %s\n", fI(N[0], 8).c_str());
    else if (D == 2) fprintf(f1, " No. of space steps NX = %s, NY = %s\n", fI(N[0], 8).c_str(), fI(N[1], 8).c_str());
    else fprintf(f1, " No. of space steps NX = %s, NY = %s, NZ = %s\n", fI(N[0], 8).c_str(), fI(N[1], 8).c_str(), fI(N[2], 8).c_str());
    fprintf(f1, " No. of time steps : NITER = %s, NSTP = %s, STP = %s\n", fI(NITER, 9).c_str(), fI(NSTP, 9).c_str(),
            fI(STP, D == 1 ? 7 : 9).c_str());
    if (D == 1) {
        fprintf(f1, " Space Step DX = %s\n", fF(DX[0], 10, 6).c_str());
        fprintf(f1, " Time Step  DT = %s, MAG =%s\n", fF(DT, 10, 6).c_str(), fF(MAG, 12, 6).c_str());
    } else if (D == 2) {
        fprintf(f1, " Space Step DX = %s, DY = %s\n", fF(DX[0], 10, 6).c_str(), fF(DX[1], 10, 6).c_str());
        fprintf(f1, " Time Step  DT = %s, MAG = %s\n", fF(DT, 10, 6).c_str(), fF(MAG, 12, 6).c_str());
    } else {
        fprintf(f1, " Spatial step-size DX = %s, DY = %s, DZ = %s\n", fF(DX[0], 10, 6).c_str(), fF(DX[1], 10, 6).c_str(),
                fF(DX[2], 10, 6).c_str());
        fprintf(f1, " Temporal step-size  DT = %s, MAG = %s\n", fF(DT, 10, 6).c_str(), fF(MAG, 12, 6).c_str());
    }
    fprintf(f1, " \n");
    fprintf(f1, " AOSC = %s\n", fE(AOSC, 12, 4).c_str());
    if (SPIN == 1) {
        if (D == 3) {
            fprintf(f1, " A0 = %s, A2 = %s (all in units of Bohr radius)\n", fF(A0, 12, 6).c_str(), fF(A2, 12, 6).c_str());
            fprintf(f1, " TAU(0) = %s, TAU(1) = %s in dimensionless units \n", fF(TAU[0] / 2, 12, 6).c_str(),
                    fF(TAU[1] / 2, 12, 6).c_str());
        } else {
            fprintf(f1, " A0 = %s, A2 = %s,  (all in units of Bohr radius) \n", fF(A0, 12, 6).c_str(), fF(A2, 12, 6).c_str());
            fprintf(f1, " TAU(0) = %s, TAU(1) = %s (in dimensionless units)\n", fF(TAU[0] / 2, 12, 6).c_str(),
                    fF(TAU[1] / 2, 12, 6).c_str());
        }
    } else {
        fprintf(f1, " A0 = %s, A2 = %s, A4 = %s (all in units of Bohr radius) \n", fF(A0, 12, 6).c_str(),
                fF(A2, 12, 6).c_str(), fF(A4, 12, 6).c_str());
        fprintf(f1, " TAU(0) = %s, TAU(1) = %s, TAU(2) = %s (in dimensionless units)\n", fF(TAU[0] / 2, 12, 6).c_str(),
                fF(TAU[1] / 2, 12, 6).c_str(), fF(TAU[2] / 2, 12, 6).c_str());
    }
    fprintf(f1, " \n");

    // ---------------------------------------------- INITIALIZE
    // grids (cgpe1d.f90:692-704), guesses (cgpe1d.f90:707-790,
    // cgpe2d.f90:689-776, cgpe3d.f90:747-837) with the reference's TF typos
    const long long NP = (long long)N[0] * N[1] * N[2];
    std::vector<double> X[3];
    for (int a = 0; a < 3; ++a) {
        X[a].assign(N[a], 0.0);
        if (a < D) {
            const double L = N[a] * DX[a];
            for (int i = 1; i <= N[a]; ++i) X[a][i - 1] = (-1.0 + 2.0 * (i - 1.0) / N[a]) * L / 2.0;
        }
    }
    std::vector<cd> phi((size_t)NP * MS);
    const double nrm = D == 1 ? sqrt(sqrt(PI)) : D == 2 ? sqrt(PI) : pow(PI, 0.75);
    for (int k = 0; k < N[2]; ++k)
        for (int j = 0; j < N[1]; ++j)
            for (int i = 0; i < N[0]; ++i) {
                const long long t = i + (long long)N[0] * (j + (long long)N[1] * k);
                const double x2 = X[0][i] * X[0][i], y2 = X[1][j] * X[1][j], z2 = X[2][k] * X[2][k];
                double tmp = ALPHAX * x2, vv = ALPHAX * ALPHAX * x2;
                if (D >= 2) { tmp += ALPHAY * y2; vv += ALPHAY * ALPHAY * y2; }
                if (D >= 3) { tmp += ALPHAZ * z2; vv += ALPHAZ * ALPHAZ * z2; }
                const double g = exp(-tmp / 2.0) / nrm;
                double p[5] = {0, 0, 0, 0, 0};
                if (SPIN == 1) {
                    if (OPTION_FPC == 1) {
                        double tf, f;
                        if (D == 1) {
                            const double base = 3.0 * (TAU[0] + TAU[2]) / 4.0;
                            const double r = pow(base, 0.67) - vv;
                            tf = r >= 0 ? r / (TAU[0] + TAU[2]) : 0.0;
                            f = pow(base, 0.33) >= 10.0 ? sqrt(tf) : g;
                        } else if (D == 2) {
                            const double base = 4.0 * (TAU[0] + TAU[1]) / (2.0 * PI);
                            const double r = pow(base, 8.0) - vv;
                            tf = r >= 0 ? (pow(base, 0.5) - vv) / (TAU[0] + TAU[1]) : 0.0;
                            f = pow(base, 0.25) >= 10.0 ? sqrt(tf) : g;
                        } else {
                            const double base = 15.0 * (TAU[0] + TAU[1]) / (8.0 * PI);
                            const double r = pow(base, 0.4) - vv;
                            tf = r >= 0 ? r / (TAU[0] + TAU[1]) : 0.0;
                            f = pow(base, 0.2) >= 10.0 ? sqrt(tf) : g;
                        }
                        p[0] = ((1.0 + MAG) / 2.0) * f; p[1] = sqrt((1.0 - MAG * MAG) / 2.0) * f; p[2] = ((1.0 - MAG) / 2.0) * f;
                    } else if (OPTION_FPC == 2) {
                        p[0] = sqrt((1.0 + MAG) / 2.0) * g; p[2] = sqrt((1.0 - MAG) / 2.0) * g;
                    } else {
                        const double gg = D == 3 ? exp(-(x2 + y2 + z2) / 2.0) / pow(PI, 0.75) : g;
                        p[0] = p[1] = p[2] = gg;
                    }
                } else {
                    if (OPTION_FPC == 1) {
                        double f;
                        if (D == 1) {
                            const double base = 3.0 * (TAU[0] + 4.0 * TAU[1]) / 4.0;
                            const double r = pow(base, 0.67) - vv;
                            const double tf = r >= 0 ? r / (TAU[0] + 4.0 * TAU[1]) : 0.0;
                            f = (3.0 * pow(TAU[0] + 4.0 * TAU[1] / 4.0, 0.33)) >= 10.0 ? sqrt(tf) : g;
                        } else if (D == 2) {
                            const double base = 4.0 * (TAU[0] + 4.0 * TAU[1]) / (2.0 * PI);
                            const double r = pow(base, 0.5) - vv;
                            const double tf = r >= 0 ? r / (TAU[0] + 4.0 * TAU[1]) : 0.0;
                            f = pow(base, 0.25) >= 10.0 ? sqrt(tf) : g;
                        } else {
                            const double base = 15.0 * (TAU[0] + 4.0 * TAU[1]) / (8.0 * PI);
                            const double r = pow(base, 0.4) - vv;
                            const double tf = r >= 0 ? r / (TAU[0] + 4.0 * TAU[1]) : 0.0;
                            f = pow(4.0 * (TAU[0] + 4.0 * TAU[1]) / (2.0 * PI), 0.25) >= 10.0 ? sqrt(tf) : g;
                        }
                        p[0] = ((2.0 + MAG) * (2.0 + MAG) / 16.0) * f;
                        p[1] = ((sqrt(4.0 - MAG * MAG) * (2.0 + MAG)) / 8.0) * f;
                        p[2] = ((sqrt(1.5) * (4.0 - MAG * MAG)) / 8.0) * f;
                        p[3] = ((sqrt(4.0 - MAG * MAG) * (2.0 - MAG)) / 8.0) * f;
                        p[4] = ((2.0 - MAG) * (2.0 - MAG) / 16.0) * f;
                    } else if (OPTION_FPC == 2) {
                        p[0] = (sqrt(2.0 + MAG) / 2.0) * g; p[4] = (sqrt(2.0 - MAG) / 2.0) * g;
                    } else if (OPTION_FPC == 3) {
                        p[0] = sqrt((1.0 + MAG) / 3.0) * g; p[3] = sqrt((2.0 - MAG) / 3.0) * g;
                    } else {
                        const double a = D == 3 ? 1.0 : sqrt(0.2);
                        for (int m = 0; m < 5; ++m) p[m] = a * g;
                    }
                }
                for (int m = 0; m < MS; ++m) phi[t + m * NP] = p[m];
            }

    // real time: initial solution (density, phase), cgpe1d.f90:369-392,
    // cgpe2d.f90:374-399, cgpe3d.f90:383-410 (X/Y printed later are the ones
    // read back from the file)
    std::vector<double> XP = X[0], YP = X[1];
    if (SWITCH_IM != 1) {
        if (!finit) {
            const std::string a = std::string("Check if the \"initial_sol_spin") + sid + ".dat\" is available" + (D == 1 ? "?" : "");
            const std::string b = std::string("if not, user can read the \"solution_file_im_spin") + sid + ".dat\" file as an initial solution.";
            fprintf(ferr, " %s\n %s\n", a.c_str(), b.c_str());
            printf(" %s\n %s\n", a.c_str(), b.c_str());
            fclose(ferr);
            return 0;
        }
        Reader ri{finit};
        const int nv = 4 * SPIN + 2;
        for (int i = 0; i < N[0]; ++i)
            for (int j = 0; j < N[1]; ++j)
                for (int k = 0; k < N[2]; ++k) {
                    const int lead = D == 1 ? 1 : D == 2 ? 2 : 0;
                    if (!ri.read(v, lead + nv)) stop_with("error reading the initial solution file");
                    if (D >= 1 && lead >= 1) XP[i] = v[0];
                    if (lead >= 2) YP[j] = v[1];
                    const long long t = i + (long long)N[0] * (j + (long long)N[1] * k);
                    for (int m = 0; m < MS; ++m)
                        phi[t + m * NP] = sqrt(v[lead + 2 * m]) * std::exp(cd(0.0, v[lead + 2 * m + 1]));
                }
        fclose(finit);
    }

    // ---------------------------------------------- device handle
    fgpe_params prm;
    memset(&prm, 0, sizeof prm);
    prm.dim = D; prm.spin = SPIN; prm.nx = N[0]; prm.ny = N[1]; prm.nz = N[2];
    prm.dx = DX[0]; prm.dy = DX[1]; prm.dz = DX[2]; prm.dt = DT; prm.imag_time = SWITCH_IM == 1;
    for (int a = 0; a < 3; ++a) { prm.tau[a] = TAU[a]; prm.gamma[a] = G[a]; prm.alpha[a] = AL[a]; }
    const char* pe = getenv("FGPE_PRECISION");
    prm.precision = (pe && (!strcmp(pe, "fp32") || !strcmp(pe, "FP32"))) ? FGPE_FP32 : FGPE_FP64;
    prm.mag = MAG;
    fgpe_t* h = nullptr;
    check(fgpe_create(&prm, &h), nullptr);
    check(fgpe_set_state(h, (const double*)phi.data()), h);
    if (SWITCH_IM == 1) check(fgpe_normalize(h, nullptr), h);   // cgpe1d.f90:394

    std::vector<double> norm(MS), rms(MS), mu(MS), cen(2 * MS);
    double en = 0, mz = 0;
    auto observe = [&]() { check(fgpe_observables(h, &en, mu.data(), &mz, rms.data()), h); };
    auto center_abs = [&](std::vector<double>& out) {
        check(fgpe_center(h, cen.data()), h);
        out.resize(MS);
        for (int m = 0; m < MS; ++m) out[m] = hypot(cen[2 * m], cen[2 * m + 1]);
    };
    check(fgpe_norms(h, norm.data()), h);
    observe();
    auto sum = [](const std::vector<double>& a) { double s = 0; for (double x : a) s += x; return s; };

    // table header and the initial row (cgpe1d.f90:402-422, 2D/3D variants)
    std::string sep = SPIN == 1 ? std::string(23, ' ') + std::string(D == 3 ? 74 : 76, '-')
                                : std::string(22, ' ') + std::string(117, '-');
    std::string hdr;
    if (SPIN == 1)
        hdr = std::string(23, ' ') + "Norm       EN       MU1       MU2       MU3      phi1      phi2      phi3";
    else if (D == 1)
        hdr = std::string(23, ' ') + "Norm       EN       MU1       MU2       MU3       MU4       MU5       phi1      phi2      phi3     phi4      phi5";
    else if (D == 2)
        hdr = std::string(23, ' ') + "Norm       EN       MU1       MU2       MU3       MU4       MU5       phi1       phi2     phi3     phi4     phi5";
    else
        hdr = std::string(23, ' ') + "Norm       EN       MU1       MU2       MU3       MU4       MU5       phi1       phi2     phi3     phi4      phi5";
    fprintf(f1, "%s\n%s\n%s\n", sep.c_str(), hdr.c_str(), sep.c_str());
    std::vector<double> pc;
    center_abs(pc);
    {
        std::string row = SPIN == 1 ? std::string("Initial: ") + std::string(8, ' ') : std::string("Initial : ") + std::string(7, ' ');
        row += fF(sum(norm), 11, 4) + fF(en / 2.0, 10, 5);
        for (int m = 0; m < MS; ++m) row += fF(mu[m] / 2.0, 10, 5);
        for (int m = 0; m < MS; ++m) row += fF(pc[m], 10, 5);
        fprintf(f1, "%s\n", row.c_str());
    }
    auto row2 = [&](double t) {
        std::string s = fF(t, 14, 6) + fF(en / 2.0, 18, 10);
        for (int m = 0; m < MS; ++m) s += fF(rms[m], 18, 10);
        fprintf(f2, "%s\n", s.c_str());
    };
    auto row3 = [&](double t) {
        std::string s = fF(t, 14, 6);
        for (int m = 0; m < MS; ++m) s += fF(norm[m], 18, 10);
        s += fF(sum(norm), 18, 10) + fF(mz, 18, 10);
        fprintf(f3, "%s\n", s.c_str());
    };
    row2(0.0);
    row3(0.0);

    // ---------------------------------------------- solution writers
    std::vector<double> st((size_t)NP * MS * 2);
    auto fetch = [&]() { check(fgpe_get_state(h, st.data()), h); };
    auto rho_th = [&](long long t, int m, double& r, double& th) {
        const double re = st[2 * (t + m * NP)], imv = st[2 * (t + m * NP) + 1];
        r = re * re + imv * imv;
        th = atan2(imv, re);
    };
    auto write_solution = [&](FILE* f, bool tmp) {
        fetch();
        double r, th;
        if (D == 1) {
            for (int i = 0; i < N[0]; ++i) {
                std::string s = fF(XP[i], 11, 5);
                for (int m = 0; m < MS; ++m) { rho_th(i, m, r, th); s += fF(r, tmp ? 14 : 18, tmp ? 6 : 10) + fF(th, tmp ? 14 : 18, tmp ? 6 : 10); }
                fprintf(f, "%s\n", s.c_str());
            }
        } else if (D == 2) {
            for (int i = 0; i < N[0]; ++i) {
                for (int j = 0; j < N[1]; ++j) {
                    const long long t = i + (long long)N[0] * j;
                    std::string s = fF(XP[i], 8, 2) + fF(YP[j], 8, 2);
                    for (int m = 0; m < MS; ++m) { rho_th(t, m, r, th); s += fF(r, 10, 5) + fF(th, 10, 5); }
                    fprintf(f, "%s\n", s.c_str());
                }
                fprintf(f, "\n");
            }
        } else {
            for (int i = 0; i < N[0]; ++i)
                for (int j = 0; j < N[1]; ++j)
                    for (int k = 0; k < N[2]; ++k) {
                        const long long t = i + (long long)N[0] * (j + (long long)N[1] * k);
                        std::string s;
                        for (int m = 0; m < MS; ++m) { rho_th(t, m, r, th); s += fF(r, 16, 10) + fF(th, 16, 10); }
                        fprintf(f, "%s\n", s.c_str());
                    }
        }
    };
    auto write_slices = [&]() {
        // 3D transient xy / xz slices at the grid centre (cgpe3d.f90:545-565)
        double r, th;
        FILE* fxy = fopen((std::string("./OUTPUT/tmp_solution_file_spin") + sid + "_xy.dat").c_str(), "w");
        for (int i = 0; i < N[0]; ++i) {
            for (int j = 0; j < N[1]; ++j) {
                const long long t = i + (long long)N[0] * (j + (long long)N[1] * (N[2] / 2));
                std::string s = fF(X[0][i], 10, 4) + fF(X[1][j], 10, 4);
                for (int m = 0; m < MS; ++m) { rho_th(t, m, r, th); s += fF(r, 14, 8) + fF(th, 14, 8); }
                fprintf(fxy, "%s\n", s.c_str());
            }
            fprintf(fxy, "\n");
        }
        fclose(fxy);
        FILE* fxz = fopen((std::string("./OUTPUT/tmp_solution_file_spin") + sid + "_xz.dat").c_str(), "w");
        for (int i = 0; i < N[0]; ++i) {
            for (int k = 0; k < N[2]; ++k) {
                const long long t = i + (long long)N[0] * ((N[1] / 2) + (long long)N[1] * k);
                std::string s = fF(X[0][i], 10, 4) + fF(X[2][k], 10, 4);
                for (int m = 0; m < MS; ++m) { rho_th(t, m, r, th); s += fF(r, 14, 8) + fF(th, 14, 8); }
                fprintf(fxz, "%s\n", s.c_str());
            }
            fprintf(fxz, "\n");
        }
        fclose(fxz);
    };
    auto after_row = [&](const std::string& lead) {
        std::vector<double> c;
        center_abs(c);
        std::string s = lead + fF(sum(norm), 7, 4);
        std::vector<double> vals;
        vals.push_back(en / 2.0);
        for (int m = 0; m < MS; ++m) vals.push_back(mu[m] / 2.0);
        for (int m = 0; m < MS; ++m) vals.push_back(c[m]);
        for (double x : vals) s += fF(x, 10, 5);
        fprintf(f1, "%s\n", s.c_str());
    };

    // ---------------------------------------------- time loop
    double en_old = en;
    long long ii = 0;
    bool exited = false;
    while (ii < NITER) {
        long long nxt = std::min<long long>(NITER, (ii / STP + 1) * STP);
        if (NSTP > 0) nxt = std::min<long long>(nxt, (ii / NSTP + 1) * NSTP);
        long long left = nxt - ii;
        while (left > 0) {
            const int chunk = (int)std::min<long long>(left, 1 << 20);
            check(fgpe_step(h, chunk), h);
            left -= chunk;
        }
        ii = nxt;
        check(fgpe_norms(h, norm.data()), h);
        if (ii % STP == 0) {
            observe();
            if (SWITCH_IM == 1) {
                double dphi = 0;
                check(fgpe_conv(h, &dphi), h);
                const double conv = dphi / (STP * 2.0 * DT);
                // EN_OLD starts at 0 and takes EN after every step
                // (cgpe1d.f90:294, 507): only a boundary at II = 1 sees the 0
                const double conv_en = fabs(en - (ii > 1 ? en_old : 0.0)) / (STP * 2.0 * DT);
                fprintf(f9, "%s%s%s\n", fList(2.0 * ii * DT).c_str(), fList(conv).c_str(), fList(conv_en).c_str());
                if (conv <= TOL || conv_en <= TOL) { exited = true; break; }
            }
            row2(2.0 * ii * DT);
            row3(2.0 * ii * DT);
            en_old = en;
        }
        if (NSTP > 0 && ii % NSTP == 0) {
            after_row(D == 3 ? "After NSTP iter.:    " : "After NSTP iter.    :");
            FILE* f7 = fopen((std::string("./OUTPUT/tmp_solution_file_spin") + sid + ".dat").c_str(), "w");
            write_solution(f7, D == 1);
            fclose(f7);
            if (D == 3) write_slices();
        }
        fflush(f1); fflush(f2); fflush(f3);
        if (f9) fflush(f9);
    }
    const long long ii_report = exited ? ii - 1 : NITER;   // II-1 (cgpe1d.f90:531)

    // ---------------------------------------------- final output
    observe();
    fprintf(f1, "%s\n", sep.c_str());
    after_row("After " + fI(ii_report, 8) + " iter.:");
    fprintf(f1, "%s\n", sep.c_str());
    fprintf(f1, " \n");
    write_solution(f8, false);
    fclose(f8);
    fgpe_destroy(h);
    printf(" Program execution complete\n");
    date_line(f1, "Ended");
    fprintf(f1, "Time elapsed = %s in seconds\n", fF(wall() - t_start, 18, D == 1 ? 6 : 8).c_str());
    fclose(f1); fclose(f2); fclose(f3);
    if (f9) fclose(f9);
    fclose(ferr);
    return 0;
}
