/*
 * bgk_thermal -- the reference's STEP_7 program (STEP_7/main.f90) on top of
 * libbgkpcm.  It reads the same input.dat, runs the same time loop and writes
 * the same files in the working directory:
 *   fort.64                   field_check: it, mean rho, T, phi (e16.8)
 *   fort.69                   diag: beta_gras, grav, Gr, dT, Pr, Ra, Fo, theta
 *   non-dim_bulk_numbers.dat  diag: it, theta, Nusselt numbers, melt ...
 *   fort.666 / .667 / .668    probe, x-profile (row Ny/2), y-profile (col Nx/2)
 *   log.dat, Nusselt.dat, Output_XXXXXXXX.vtk (ASCII structured grid)
 * The host is C++ because no Fortran compiler is available to build the
 * reference's own main.f90 against the C ABI (the binding a Fortran host
 * would use is bgk_pcm_b200/fortran/bgk_c.f90).
 *
 * usage: bgk_thermal [dir] [--precision f64|f32|f16|f32x] [--fma] [--tanh portable|device]
 *                    [--heat west|right|bottom|right+bottom]
 *                    [--snapshot-in file] [--snapshot-out file] [--dump-out]
 * --heat selects the heated wall of the reference's STEP_DOCONCURRENT build
 * options (right = FROMRIGHT, bottom = FROMBOTTOM, both = both macros).
 * dump != 0 in input.dat restarts from the reference's text dump
 * (dumpFile.dat, plus dumpPhi.dat when present); --dump-out writes both at
 * the end of the run.
 */
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <chrono>
#include <sys/resource.h>

#include "bgk_pcm.h"

namespace {

struct Ctx {
    bgk_ctx *h = nullptr;
    bgk_params p{};
    std::string dir;
    int Nx = 0, Ny = 0;
    FILE *u64 = nullptr, *u69 = nullptr, *u164 = nullptr, *u666 = nullptr, *u667 = nullptr, *u668 = nullptr;
    double melt_front = 0.0, melt_front_expected = 0.0;   /* diag.f90 locals kept across calls */
};

void die(const char *what, int rc)
{
    fprintf(stderr, "bgk_thermal: %s failed (%d): %s\n", what, rc, bgk_last_error());
    exit(1);
}

#define CALL(x)                        \
    do {                               \
        int rc_ = (x);                 \
        if (rc_ != BGK_OK) die(#x, rc_); \
    } while (0)

/* Fortran Ew.d: 0.ddddddE+xx right-justified in w (3-digit exponents drop the E). */
std::string fE(double x, int w, int d)
{
    char body[96];
    if (x == 0.0 || !std::isfinite(x)) {
        if (x == 0.0) snprintf(body, sizeof body, "0.%0*dE+00", d, 0);
        else snprintf(body, sizeof body, "%s", std::isnan(x) ? "NaN" : (x > 0 ? "Infinity" : "-Infinity"));
    } else {
        char tmp[64];
        snprintf(tmp, sizeof tmp, "%.*e", d - 1, std::fabs(x));
        const char *e = strchr(tmp, 'e');
        int ex = atoi(e + 1) + 1;
        std::string digits;
        for (const char *c = tmp; c < e; c++)
            if (*c >= '0' && *c <= '9') digits.push_back(*c);
        if (ex >= -99 && ex <= 99)
            snprintf(body, sizeof body, "%s0.%sE%c%02d", x < 0 ? "-" : "", digits.c_str(), ex < 0 ? '-' : '+', std::abs(ex));
        else
            snprintf(body, sizeof body, "%s0.%s%c%03d", x < 0 ? "-" : "", digits.c_str(), ex < 0 ? '-' : '+', std::abs(ex));
    }
    std::string s(body);
    if ((int)s.size() < w) s = std::string(w - s.size(), ' ') + s;
    return s;
}

/* gfortran list-directed REAL(8) (17 significant digits). */
std::string flist(double x)
{
    char out[96];                    /* room for tmp (64) plus the exponent */
    double ax = std::fabs(x);
    if (x != 0.0 && (ax < 0.1 || ax >= 1e16)) {
        char tmp[64];
        snprintf(tmp, sizeof tmp, "%.16E", x);
        char *e = strchr(tmp, 'E');
        int ex = atoi(e + 1);
        *e = 0;
        snprintf(out, sizeof out, "%sE%c%03d", tmp, ex < 0 ? '-' : '+', std::abs(ex));
    } else {
        int intdig = ax >= 1.0 ? (int)std::floor(std::log10(ax)) + 1 : 0;
        int frac = intdig > 0 ? 17 - intdig : 17;
        if (frac < 0) frac = 0;
        snprintf(out, sizeof out, "%.*f", frac, x);
    }
    return out;
}

FILE *open_unit(const Ctx &c, const char *name, const char *mode)
{
    std::string path = c.dir + "/" + name;
    FILE *f = fopen(path.c_str(), mode);
    if (!f) {
        fprintf(stderr, "bgk_thermal: cannot open %s\n", path.c_str());
        exit(1);
    }
    return f;
}

std::vector<double> region(Ctx &c, int field, int i0, int j0, int ni, int nj)
{
    std::vector<double> v((size_t)ni * nj);
    CALL(bgk_download_region(c.h, field, i0, j0, ni, nj, v.data(), ni));
    return v;
}

int get_it(Ctx &c)
{
    int it = 0;
    CALL(bgk_get_it(c.h, &it));
    return it;
}

/* STEP_7/diag.f90:15-116 */
void diag(Ctx &c)
{
    const bgk_params &p = c.p;
    const int Nx = c.Nx, Ny = c.Ny, it = get_it(c);
    const double kvisc = (1.0 / 3.0) * (p.tau_f - 0.5);
    const double alpha = (1.0 / 3.0) * (p.tau_g - 0.5);
    const double Delta_Temp = p.T0 - p.T_in_sol;
    const double Tin = p.T0;
    const double beta_gras = (p.rho0 / p.rho1 - 1.0) / Delta_Temp;
    const int32_t ny3 = (int32_t)((uint32_t)Ny * (uint32_t)Ny * (uint32_t)Ny); /* default INTEGER wraps */
    const double Gras = p.grav * beta_gras * Delta_Temp * (double)ny3 / (kvisc * kvisc);
    const double Pr = (2.0 * p.tau_f - 1.0) / (2.0 * p.tau_g - 1.0);
    const double Ray = Pr * Gras;
    const double Fou = alpha * (double)it / (double)(Ny * Ny);
    const double theta = p.stefan_number * Fou;
    const double theta1 = std::pow(Ray, -0.5);
    const double theta2 = (double)(Nx / Ny) * std::pow(Ray, -0.25);
    fprintf(c.u69, " beta_gras, grav, Gras, Delta_Temp, Pr, Ray, Fou, theta\n ");
    const double l69[8] = {beta_gras, p.grav, Gras, Delta_Temp, Pr, Ray, Fou, theta};
    for (double v : l69) fprintf(c.u69, " %s", flist(v).c_str());
    fprintf(c.u69, "\n ---------------------------------------------\n");
    fflush(c.u69);
    const double Nus = std::pow(2.0 * theta, -0.5) +
                       (0.35 * std::pow(Ray, 0.25) - std::pow(2.0 * theta, -0.5)) *
                           std::pow(1.0 + std::pow(0.0175 * std::pow(Ray, 0.75) * std::pow(theta, 1.5), -2.0), -0.5);
    /* wall columns i = 1..3, rows 1..Ny */
    std::vector<double> Tw = region(c, BGK_FIELD_T, 1, 1, 3, Ny);
    double Nus_comp = 0.0, Nus_comp_2 = 0.0;
    for (int j = 0; j < Ny; j++) Nus_comp = Nus_comp + (double)Ny * ((Tin - Tw[3 * j + 1]) / 2.0) / Delta_Temp;
    Nus_comp = Nus_comp / (double)Ny;
    for (int j = 0; j < Ny; j++) {
        double grad_T = std::fabs((-(3.0 * Tw[3 * j]) + 4.0 * Tw[3 * j + 1] - Tw[3 * j + 2]) / 2.0);
        Nus_comp_2 = Nus_comp_2 + (double)Ny * grad_T / Delta_Temp;
    }
    Nus_comp_2 = Nus_comp_2 / (double)Ny;
    if (it % 100 == 0) {
        double sums[4];
        int rc = bgk_field_sums(c.h, sums);
        if (rc != BGK_OK && rc != BGK_ERR_NONFINITE) die("bgk_field_sums", rc);
        double melt = sums[3] / (double)(Nx * Ny);
        if (theta <= theta1) {
            c.melt_front = (double)Ny / std::pow(2.0 * theta, -0.5);
            c.melt_front_expected = (double)Ny / Nus;
        } else if (theta > theta1 && theta < theta2) {
            /* sum of i over nodes with phi exactly 0 */
            std::vector<double> ph = region(c, BGK_FIELD_PHI, 1, 1, Nx, Ny);
            double mf = 0.0;
            for (int j = 0; j < Ny; j++)
                for (int i = 0; i < Nx; i++)
                    if (ph[(size_t)j * Nx + i] == 0.0) mf = mf + (double)(i + 1);
            c.melt_front = mf / (double)Ny;
            c.melt_front_expected = (double)Ny * theta * std::pow(Ray, 0.25);
        }
        const double v[11] = {theta, Nus, Nus_comp, Nus_comp_2, melt, c.melt_front, c.melt_front_expected,
                              Gras, Pr, Ray, Fou};
        printf(" CHECK: theta = %s\n", flist(theta).c_str());
        fprintf(c.u164, "%8d", it);
        for (double x : v) fprintf(c.u164, " %s", fE(x, 13, 6).c_str());
        fprintf(c.u164, "\n");
        fflush(c.u164);
    }
}

void row5(FILE *f, int idx, const double *v)
{
    fprintf(f, "%8d", idx);
    for (int k = 0; k < 5; k++) fprintf(f, "%s ", fE(v[k], 14, 6).c_str());
    fprintf(f, "\n");
}

const int kProbeFields[5] = {BGK_FIELD_U, BGK_FIELD_V, BGK_FIELD_RHO, BGK_FIELD_T, BGK_FIELD_PHI};

/* STEP_7/probe.f90 */
void probe(Ctx &c)
{
    double v[5];
    for (int k = 0; k < 5; k++) v[k] = region(c, kProbeFields[k], c.Nx / 2, c.Ny / 2, 1, 1)[0];
    row5(c.u666, get_it(c), v);
    fflush(c.u666);
}

/* STEP_7/prof_x.f90 (row Ny/2) and prof_y.f90 (column Nx/2) */
void profile(Ctx &c, FILE *f, bool along_x)
{
    const int n = along_x ? c.Nx : c.Ny;
    std::vector<double> cols[5];
    for (int k = 0; k < 5; k++)
        cols[k] = along_x ? region(c, kProbeFields[k], 1, c.Ny / 2, c.Nx, 1)
                          : region(c, kProbeFields[k], c.Nx / 2, 1, 1, c.Ny);
    fprintf(f, "# t=%7d\n", get_it(c));
    for (int a = 0; a < n; a++) {
        double v[5] = {cols[0][a], cols[1][a], cols[2][a], cols[3][a], cols[4][a]};
        row5(f, a + 1, v);
    }
    fprintf(f, "\n\n");
    fflush(f);
}

/* STEP_7/field_check.f90 */
void field_check(Ctx &c)
{
    double s[4];
    int rc = bgk_field_sums(c.h, s);
    if (rc != BGK_OK && rc != BGK_ERR_NONFINITE) die("bgk_field_sums", rc);
    const double n = (double)(c.Nx * c.Ny);
    fprintf(c.u64, "%8d %s %s %s \n", get_it(c), fE(s[0] / n, 16, 8).c_str(), fE(s[1] / n, 16, 8).c_str(),
            fE(s[2] / n, 16, 8).c_str());
    fflush(c.u64);
    if (rc == BGK_ERR_NONFINITE) fprintf(stderr, "bgk_thermal: warning: %s\n", bgk_last_error());
}

/* STEP_7/out2d.f90 */
void out2d(Ctx &c)
{
    const int NX2 = c.Nx + 2, NY2 = c.Ny + 2;
    std::vector<double> rho((size_t)NX2 * NY2), T(rho.size()), phi(rho.size()), u(rho.size()), v(rho.size());
    CALL(bgk_download(c.h, BGK_FIELD_RHO, rho.data(), NX2));
    CALL(bgk_download(c.h, BGK_FIELD_T, T.data(), NX2));
    CALL(bgk_download(c.h, BGK_FIELD_PHI, phi.data(), NX2));
    CALL(bgk_download(c.h, BGK_FIELD_U, u.data(), NX2));
    CALL(bgk_download(c.h, BGK_FIELD_V, v.data(), NX2));
    char name[64];
    snprintf(name, sizeof name, "Output_%08d.vtk", get_it(c));
    FILE *f = open_unit(c, name, "w");
    fprintf(f, "# vtk DataFile Version 2.0\nGriglia strutturata\nASCII\nDATASET STRUCTURED_GRID\n");
    fprintf(f, "DIMENSIONS%8d%8d%8d\n", NX2, NY2, 1);
    fprintf(f, "POINTS%15d float\n", NX2 * NY2);
    for (int l = 0; l < NY2; l++)
        for (int i = 0; i < NX2; i++) fprintf(f, "%12d%12d%12d\n", i, l, 1);
    fprintf(f, "POINT_DATA%15d\n", NX2 * NY2);
    auto scal = [&](const char *title, const std::vector<double> &a) {
        fprintf(f, "SCALARS %s float 1\nLOOKUP_TABLE default\n", title);
        for (double x : a) fprintf(f, "   %s     \n", flist(x).c_str());
    };
    scal("DENSITY", rho);
    scal("Temperature", T);
    scal("Phase_Field", phi);
    fprintf(f, "VECTORS VELOCITY float\n");
    for (size_t q = 0; q < u.size(); q++)
        fprintf(f, "   %s        %s        0.0000000000000000     \n", flist(u[q]).c_str(), flist(v[q]).c_str());
    fclose(f);
}

/* The 22 arrays of the reference's text restart, in the order of one node's
 * two records (STEP_7/dump_out.f90:10-17). */
const int kDumpFields[22] = {BGK_FIELD_U, BGK_FIELD_V, BGK_FIELD_RHO,
                             BGK_FIELD_F0 + 0, BGK_FIELD_F0 + 1, BGK_FIELD_F0 + 2, BGK_FIELD_F0 + 3,
                             BGK_FIELD_F0 + 4, BGK_FIELD_F0 + 5, BGK_FIELD_F0 + 6, BGK_FIELD_F0 + 7,
                             BGK_FIELD_F0 + 8, BGK_FIELD_T,
                             BGK_FIELD_G0 + 0, BGK_FIELD_G0 + 1, BGK_FIELD_G0 + 2, BGK_FIELD_G0 + 3,
                             BGK_FIELD_G0 + 4, BGK_FIELD_G0 + 5, BGK_FIELD_G0 + 6, BGK_FIELD_G0 + 7,
                             BGK_FIELD_G0 + 8};

/* gfortran list-directed item: one blank, then the value right-justified in
 * 25 columns (G25.17E3: F form followed by 5 blanks, or E form). */
std::string fitem(double x)
{
    std::string v = flist(x);
    if (v.find('E') == std::string::npos) v += "     ";
    if (v.size() < 25) v = std::string(25 - v.size(), ' ') + v;
    return " " + v;
}

/* STEP_7/dump_out.f90: dumpFile.dat with it and, for every node (i fastest,
 * halos included), u v rho f0..f8 on one record and T g0..g8 on the next.
 * The reference's file omits phi; it is written to dumpPhi.dat (one value
 * per record, same node order) so that a restart can restore it. */
void dump_out(Ctx &c)
{
    const int NX2 = c.Nx + 2, NY2 = c.Ny + 2;
    const size_t A = (size_t)NX2 * NY2;
    std::vector<double> a(22 * A), phi(A);
    for (int k = 0; k < 22; k++) CALL(bgk_download(c.h, kDumpFields[k], a.data() + k * A, NX2));
    CALL(bgk_download(c.h, BGK_FIELD_PHI, phi.data(), NX2));
    FILE *f = open_unit(c, "dumpFile.dat", "w");
    fprintf(f, " %11d\n", get_it(c));
    std::string line;
    for (size_t q = 0; q < A; q++) {
        line.clear();
        for (int k = 0; k < 12; k++) line += fitem(a[k * A + q]);
        line += "\n";
        for (int k = 12; k < 22; k++) line += fitem(a[k * A + q]);
        line += "\n";
        fputs(line.c_str(), f);
    }
    fclose(f);
    FILE *fp = open_unit(c, "dumpPhi.dat", "w");
    for (size_t q = 0; q < A; q++) fprintf(fp, "%s\n", fitem(phi[q]).c_str());
    fclose(fp);
}

/* Next real of a list-directed file (E or D exponents). */
bool read_real(FILE *f, double *x)
{
    char tok[128];
    if (fscanf(f, "%127s", tok) != 1) return false;
    for (char *p = tok; *p; p++)
        if (*p == 'D' || *p == 'd') *p = 'E';
    char *end = nullptr;
    *x = strtod(tok, &end);
    return end && *end == 0;
}

/* STEP_7/dump_in.f90 for dump != 0: the state of dumpFile.dat (and phi from
 * dumpPhi.dat when present) over a fresh initial condition. */
int dump_in(Ctx &c)
{
    const int NX2 = c.Nx + 2, NY2 = c.Ny + 2;
    const size_t A = (size_t)NX2 * NY2;
    std::string path = c.dir + "/dumpFile.dat";
    FILE *f = fopen(path.c_str(), "r");
    if (!f) {
        fprintf(stderr, "bgk_thermal: dump = %d but %s cannot be opened\n", c.p.dump, path.c_str());
        exit(1);
    }
    double itd = 0.0;
    if (!read_real(f, &itd)) {
        fprintf(stderr, "bgk_thermal: %s: no iteration count\n", path.c_str());
        exit(1);
    }
    std::vector<double> a(22 * A);
    for (size_t q = 0; q < A; q++)
        for (int k = 0; k < 22; k++)
            if (!read_real(f, &a[k * A + q])) {
                fprintf(stderr, "bgk_thermal: %s ends early (node %zu of %zu)\n", path.c_str(), q, A);
                exit(1);
            }
    fclose(f);
    CALL(bgk_initialize(c.h));
    for (int k = 0; k < 22; k++) CALL(bgk_upload(c.h, kDumpFields[k], a.data() + k * A, NX2));
    std::string ppath = c.dir + "/dumpPhi.dat";
    FILE *fp = fopen(ppath.c_str(), "r");
    if (fp) {
        std::vector<double> phi(A);
        for (size_t q = 0; q < A; q++)
            if (!read_real(fp, &phi[q])) {
                fprintf(stderr, "bgk_thermal: %s ends early\n", ppath.c_str());
                exit(1);
            }
        fclose(fp);
        CALL(bgk_upload(c.h, BGK_FIELD_PHI, phi.data(), NX2));
    } else {
        fprintf(stderr, "bgk_thermal: %s not found: phi keeps the initial condition (the reference's "
                        "dumpFile.dat does not hold phi)\n", ppath.c_str());
    }
    const int it = (int)itd;
    CALL(bgk_set_it(c.h, it));
    return it;
}

double get_mem_mb()
{
    struct rusage r;
    getrusage(RUSAGE_SELF, &r);
    return (double)r.ru_maxrss / 1024.0;
}

} // namespace

int main(int argc, char **argv)
{
    Ctx c;
    c.dir = ".";
    bgk_options opt{BGK_PREC_F64, BGK_TANH_PORTABLE, 0, -1, 0, BGK_HEAT_WEST};
    std::string snap_in, snap_out;
    bool dump_at_end = false;
    for (int a = 1; a < argc; a++) {
        std::string s = argv[a];
        if (s == "--precision" && a + 1 < argc) {
            std::string v = argv[++a];
            opt.precision = v == "f32" ? BGK_PREC_F32
                          : (v == "f16" ? BGK_PREC_F16 : (v == "f32x" ? BGK_PREC_F32X : BGK_PREC_F64));
        } else if (s == "--fma") {
            opt.fma = 1;
        } else if (s == "--tanh" && a + 1 < argc) {
            opt.tanh_mode = std::string(argv[++a]) == "device" ? BGK_TANH_DEVICE : BGK_TANH_PORTABLE;
        } else if (s == "--heat" && a + 1 < argc) {
            const std::string v = argv[++a];
            opt.heat = (v.find("right") != std::string::npos ? BGK_HEAT_RIGHT : 0) |
                       (v.find("bottom") != std::string::npos ? BGK_HEAT_BOTTOM : 0);
            if (opt.heat == 0 && v != "west") {
                fprintf(stderr, "bgk_thermal: --heat takes west, right, bottom or right+bottom\n");
                return 1;
            }
            printf(" Heating from %s\n", (opt.heat & BGK_HEAT_RIGHT) ? "right (Est wall)" : "left (West wall)");
        } else if (s == "--snapshot-in" && a + 1 < argc) {
            snap_in = argv[++a];
        } else if (s == "--snapshot-out" && a + 1 < argc) {
            snap_out = argv[++a];
        } else if (s == "--dump-out") {
            dump_at_end = true;
        } else {
            c.dir = s;
        }
    }
    printf(" ====================================\n B200 fused version (libbgkpcm)\n ====================================\n");
    CALL(bgk_read_input((c.dir + "/input.dat").c_str(), &c.p));
    c.Nx = c.p.Nx;
    c.Ny = c.p.Ny;
    if (c.p.noutput <= 0) {
        fprintf(stderr, "bgk_thermal: noutput must be positive\n");
        return 1;
    }
    CALL(bgk_create(&c.p, &opt, &c.h));
    int it = 0;
    if (!snap_in.empty()) {
        CALL(bgk_load(c.h, snap_in.c_str()));
        it = get_it(c);
    } else if (c.p.dump != 0) {
        it = dump_in(c);
    } else {
        CALL(bgk_initialize(c.h));
        FILE *lg = open_unit(c, "log.dat", "w");
        fprintf(lg, " iteration    mass\n ====================\n");
        fclose(lg);
    }
    const int it0 = it + 1;
    const int deltaOut = c.p.iter / c.p.noutput;
    int itOut;
    if (it == 0) {
        itOut = deltaOut;
        out2d(c);
    } else {
        itOut = it + deltaOut;
    }
    c.u64 = open_unit(c, "fort.64", "w");
    c.u69 = open_unit(c, "fort.69", "w");
    c.u164 = open_unit(c, "non-dim_bulk_numbers.dat", "w");
    c.u666 = open_unit(c, "fort.666", "w");
    c.u667 = open_unit(c, "fort.667", "w");
    c.u668 = open_unit(c, "fort.668", "w");
    printf("INFO: Memory used (MB)      %14.6f \n", get_mem_mb());
    auto t0 = std::chrono::steady_clock::now();
    it = it0 - 1;
    while (it < c.p.iter) {
        /* advance to the next step at which the reference produces output */
        int next = c.p.iter;
        int nd = (it / 1000 + 1) * 1000;
        if (nd < next) next = nd;
        if (itOut > it && itOut < next) next = itOut;
        CALL(bgk_step(c.h, next - it));
        it = next;
        if (it % 1000 == 0) {
            diag(c);
            probe(c);
            profile(c, c.u667, true);
            profile(c, c.u668, false);
            field_check(c);
            FILE *lg = open_unit(c, "log.dat", "a");
            fprintf(lg, "%8d %10.4f\n", it, 0.0); /* `mass` is never computed in STEP_7 */
            fclose(lg);
        }
        if (it == itOut || it == c.p.iter) {
            out2d(c);
            FILE *nf = open_unit(c, "Nusselt.dat", "w");
            for (int i = 1; i <= 40; i++) fprintf(nf, "%8d %10.4f %10.4f %10.4f\n", i, 0.0, 0.0, 0.0);
            fclose(nf);
            itOut = itOut + deltaOut;
        }
    }
    CALL(bgk_sync(c.h));
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const int nsteps = c.p.iter - (it0 - 1);
    printf(" ==========================================\n INFO: Run completed\n");
    printf("INFO: Main loop time        %14.6E \n", secs);
    printf("INFO: Mean time for timestep%14.6E \n", nsteps > 0 ? secs / nsteps : 0.0);
    /* the reference prints Mlups in single precision: float(nx)/1000*float(ny)/1000*(float(iter)/time) */
    const float mlups = ((float)c.Nx / 1000.0f * (float)c.Ny / 1000.0f) * ((float)nsteps / (float)secs);
    printf("INFO: Mlups                 %14.6f \n", (double)mlups);
    printf("INFO: Memory used (MB)      %14.6f \n", get_mem_mb());
    printf(" ==========================================\n");
    if (!snap_out.empty()) CALL(bgk_save(c.h, snap_out.c_str()));
    if (dump_at_end) dump_out(c);
    FILE *us[] = {c.u64, c.u69, c.u164, c.u666, c.u667, c.u668};
    for (FILE *f : us) fclose(f);
    CALL(bgk_destroy(c.h));
    return 0;
}
