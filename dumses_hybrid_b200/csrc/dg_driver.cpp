// dg_driver: the reference's main program (src/dumses.f90:37-185) over the C-ABI of
// libdumses_gpu.so, for a host language with no Fortran compiler.  It reads the same
// `input` namelist file (src/subroutines/init.f90:127-240, defaults :244-302), sets up
// the initial state (init.f90:76-122: condinit, boundary, or restart_run from a binary
// dump), writes dump 0 and the first history line, and runs the time loop of
// dumses.f90:75-160: compute_dt, godunov, fargo_update, boundary, dissipation, then
// history and output whenever time crosses the next dthist / dtdump mark, until
// time - dt > tlim.  Errors stop the run with the library's message (the Fortran shims
// `stop 1`).
//
// The reference's compile-time switches (NDIM, ISO) and its problem directory
// (condinit) are command-line options here:
//   dg_driver [input] [--ndim 2|3] [--iso 0|1] [--ic NAME] [--beta B] [--amp A] [--seed S]
//             [--precision fp64|fp32] [--nsteps N] [--out DIR] [--final-dump PATH]
//             [--quiet] [--print-params]
// NAME is one of field_loop, orszag_tang, mri, mri_test (the initial conditions of the
// library's dg_condinit).  --nsteps stops after N steps (a debugging limit, like the
// reference's debug mode stops after 5 dumps); --final-dump writes the state after the
// last step; --print-params prints the parameters read from the input file and exits
// without touching a GPU.
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "dumses_gpu.h"

namespace {

[[noreturn]] void stop(const std::string &what) {
    std::fprintf(stderr, "dg_driver: %s\n", what.c_str());
    std::exit(1);
}

void check(int rc, const char *call) {
    if (rc != DG_OK) stop(std::string(call) + " returned " + std::to_string(rc) + ": " + dg_last_error());
}

std::string lower(std::string s) {
    for (char &c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

// key = value pairs of every namelist group of a Fortran namelist file; keys lower-case,
// quotes stripped (the groups of init.f90:153-158 use distinct names)
std::map<std::string, std::string> read_namelist(const std::string &path) {
    std::ifstream f(path);
    if (!f) stop("cannot open input file " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string t = ss.str();
    std::map<std::string, std::string> kv;
    size_t i = 0;
    auto is_key = [](char c) { return std::isalnum((unsigned char)c) || c == '_'; };
    while (i < t.size()) {
        if (t[i] == '!') {  // comment to the end of the line
            while (i < t.size() && t[i] != '\n') i++;
            continue;
        }
        if (t[i] == '&') {  // group name
            i++;
            while (i < t.size() && is_key(t[i])) i++;
            continue;
        }
        if (!is_key(t[i])) {
            i++;
            continue;
        }
        size_t k0 = i;
        while (i < t.size() && is_key(t[i])) i++;
        std::string key = lower(t.substr(k0, i - k0));
        size_t j = i;
        while (j < t.size() && (t[j] == ' ' || t[j] == '\t')) j++;
        if (j >= t.size() || t[j] != '=') continue;
        j++;
        while (j < t.size() && std::isspace((unsigned char)t[j])) j++;
        std::string val;
        if (j < t.size() && (t[j] == '\'' || t[j] == '"')) {
            const char q = t[j++];
            size_t v0 = j;
            while (j < t.size() && t[j] != q) j++;
            val = t.substr(v0, j - v0);
            if (j < t.size()) j++;
        } else {
            size_t v0 = j;
            while (j < t.size() && !std::isspace((unsigned char)t[j]) && t[j] != ',' && t[j] != '/') j++;
            val = t.substr(v0, j - v0);
        }
        kv[key] = val;
        i = j;
    }
    return kv;
}

double fnum(const std::string &s) {  // Fortran real literal (d or D exponent)
    std::string c = s;
    for (char &ch : c)
        if (ch == 'd' || ch == 'D') ch = 'e';
    char *end = nullptr;
    const double v = std::strtod(c.c_str(), &end);
    if (end == c.c_str()) stop("not a number: " + s);
    return v;
}

bool flogical(const std::string &s) {  // .true. / T / .false. / F
    std::string c = lower(s);
    while (!c.empty() && c[0] == '.') c.erase(0, 1);
    return !c.empty() && c[0] == 't';
}

std::string trim(std::string s) {
    while (!s.empty() && std::isspace((unsigned char)s.back())) s.pop_back();
    size_t a = 0;
    while (a < s.size() && std::isspace((unsigned char)s[a])) a++;
    return s.substr(a);
}

int riemann_id(const std::string &name, bool two_d) {  // init_solver (init.f90:306-345)
    const std::string n = lower(trim(name));
    if (n == "llf") return DG_RIEMANN_LLF;
    if (n == "hll" && !two_d) return DG_RIEMANN_HLL;
    if (n == "hlld") return DG_RIEMANN_HLLD;
    if (n == "upwind") return DG_RIEMANN_UPWIND;
    if (n == "hlla" && two_d) return DG_RIEMANN_HLLA;
    stop("unsupported " + std::string(two_d ? "riemann2d" : "riemann") + " = '" + name + "'");
}

int bc_id(const std::string &name) {
    const std::string n = lower(trim(name));
    if (n == "periodic") return DG_BC_PERIODIC;
    if (n == "zero_gradient") return DG_BC_ZERO_GRADIENT;
    if (n == "shearingbox") return DG_BC_SHEARINGBOX;
    stop("unsupported boundary type '" + name + "'");
}

struct Run {
    dg_params p;
    int restart = 0;
    double tlim = 1.0, dtdump = -1.0, dthist = -1.0;
    bool debug = false;
    std::string io_type = "binary";
};

Run parse_input(const std::string &path, int ndim, int iso) {
    Run r;
    dg_default_params(&r.p);
    r.p.ndim = ndim;
    r.p.iso = iso;
    const auto kv = read_namelist(path);
    auto has = [&](const char *k) { return kv.count(k) > 0; };
    auto get = [&](const char *k) { return kv.at(k); };
    if (has("restart")) r.restart = (int)fnum(get("restart"));
    if (has("tlim")) r.tlim = fnum(get("tlim"));
    if (has("debug")) r.debug = flogical(get("debug"));
    if (has("dtdump")) r.dtdump = fnum(get("dtdump"));
    if (has("dthist")) r.dthist = fnum(get("dthist"));
    if (has("io_type")) r.io_type = lower(trim(get("io_type")));
    if (has("nx")) r.p.nx = (int)fnum(get("nx"));
    if (has("ny")) r.p.ny = (int)fnum(get("ny"));
    if (has("nz")) r.p.nz = (int)fnum(get("nz"));
    const char *reals[] = {"xmin", "xmax", "ymin", "ymax", "zmin", "zmax", "gamma", "ciso", "omega0", "courant", "nu", "eta"};
    double *dst[] = {&r.p.xmin, &r.p.xmax, &r.p.ymin, &r.p.ymax, &r.p.zmin, &r.p.zmax, &r.p.gamma, &r.p.ciso,
                     &r.p.omega0, &r.p.courant, &r.p.nu, &r.p.eta};
    for (int q = 0; q < 12; q++)
        if (has(reals[q])) *dst[q] = fnum(get(reals[q]));
    if (has("slope_type")) r.p.slope_type = (int)fnum(get("slope_type"));
    if (has("riemann")) r.p.iriemann = riemann_id(get("riemann"), false);
    if (has("riemann2d")) r.p.iriemann2d = riemann_id(get("riemann2d"), true);
    const char *bcs[] = {"bdtypex", "bdtypey", "bdtypez"};
    for (int d = 0; d < 3; d++)
        if (has(bcs[d])) r.p.bc[d] = bc_id(get(bcs[d]));
    if (has("fargo")) r.p.fargo = flogical(get("fargo")) ? 1 : 0;
    if (has("rhs") && flogical(get("rhs"))) stop("rhs = .true. (source terms) is outside this library's step");
    if (ndim < 3) r.p.nz = 1;
    return r;
}

// Fortran edit 1PEw.5 (one digit before the point, five after; a three-digit exponent
// drops the E), right-justified in w columns
std::string fortran_1pe(double x, int w) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.5E", x);
    std::string s = buf;
    const size_t e = s.find('E');
    if (e != std::string::npos && s.size() - e - 1 > 3) s.erase(e, 1);
    if ((int)s.size() < w) s.insert(0, (size_t)w - s.size(), ' ');
    return s;
}

// history file (src/problem/mri/history.f90:146-170; src/subroutines/history.f90:146-167 writes the
// same header and format): a header when the run starts at time 0, then one line per call
void write_history(const std::string &path, double time, double dt, const double s[9]) {
    const bool fresh = time == 0.0;
    FILE *f = std::fopen(path.c_str(), fresh ? "w" : "a");
    if (!f) stop("cannot open " + path);
    if (fresh) {
        const char *k[] = {"mass", "maxwell", "reynolds", "max+rey", "magp", "meanBx", "meanBy", "meanBz", "divB"};
        std::fprintf(f, "# %11s %12s ", "time", "dt");
        for (const char *n : k) std::fprintf(f, "%14s ", n);
        std::fprintf(f, "\n");
    }
    std::string line = " " + fortran_1pe(time, 12) + " " + fortran_1pe(dt, 12) + " ";
    for (int q = 0; q < 9; q++) line += fortran_1pe(s[q], 14) + " ";
    std::fprintf(f, "%s\n", line.c_str());
    std::fclose(f);
}

// output_NNNNNN/data.000000.bin under dir (get_filename, src/modules/file.f90; output.f90:225)
std::string dump_path(const std::string &dir, int ndump) {
    char sub[32];
    std::snprintf(sub, sizeof sub, "output_%06d", ndump % 1000000);
    const std::string d = dir + "/" + sub;
    mkdir(d.c_str(), 0755);
    return d + "/data.000000.bin";
}

int ic_id(const std::string &name) {
    if (name == "field_loop") return 1;
    if (name == "orszag_tang") return 2;
    if (name == "mri") return 3;
    if (name == "mri_test") return 4;
    stop("unknown --ic " + name);
}

}  // namespace

int main(int argc, char **argv) {
    std::string input = "input", out = ".", ic = "orszag_tang", final_dump;
    int ndim = 3, iso = 0, precision = DG_PREC_FP64;
    long long nsteps = -1;
    double beta = 1000.0, amp = 0.0;
    unsigned long long seed = 0;
    bool quiet = false, print_params = false;
    for (int a = 1; a < argc; a++) {
        const std::string s = argv[a];
        auto next = [&]() -> std::string {
            if (a + 1 >= argc) stop("missing value after " + s);
            return argv[++a];
        };
        if (s == "--ndim") ndim = std::atoi(next().c_str());
        else if (s == "--iso") iso = std::atoi(next().c_str());
        else if (s == "--ic") ic = next();
        else if (s == "--beta") beta = fnum(next());
        else if (s == "--amp") amp = fnum(next());
        else if (s == "--seed") seed = std::strtoull(next().c_str(), nullptr, 10);
        else if (s == "--precision") {
            const std::string v = next();
            if (v == "fp64") precision = DG_PREC_FP64;
            else if (v == "fp32") precision = DG_PREC_FP32;
            else stop("--precision must be fp64 or fp32");
        } else if (s == "--nsteps") nsteps = std::atoll(next().c_str());
        else if (s == "--out") out = next();
        else if (s == "--final-dump") final_dump = next();
        else if (s == "--quiet") quiet = true;
        else if (s == "--print-params") print_params = true;
        else if (!s.empty() && s[0] != '-') input = s;
        else stop("unknown option " + s);
    }
    Run r = parse_input(input, ndim, iso);
    r.p.precision = precision;
    if (print_params) {
        const dg_params &p = r.p;
        std::printf("ndim=%d iso=%d nx=%d ny=%d nz=%d\n", p.ndim, p.iso, p.nx, p.ny, p.nz);
        std::printf("xmin=%.17g xmax=%.17g ymin=%.17g ymax=%.17g zmin=%.17g zmax=%.17g\n", p.xmin, p.xmax, p.ymin,
                    p.ymax, p.zmin, p.zmax);
        std::printf("gamma=%.17g ciso=%.17g omega0=%.17g courant=%.17g nu=%.17g eta=%.17g\n", p.gamma, p.ciso,
                    p.omega0, p.courant, p.nu, p.eta);
        std::printf("slope_type=%d iriemann=%d iriemann2d=%d bc=%d,%d,%d fargo=%d\n", p.slope_type, p.iriemann,
                    p.iriemann2d, p.bc[0], p.bc[1], p.bc[2], p.fargo);
        std::printf("restart=%d tlim=%.17g dtdump=%.17g dthist=%.17g debug=%d io_type=%s\n", r.restart, r.tlim,
                    r.dtdump, r.dthist, r.debug ? 1 : 0, r.io_type.c_str());
        return 0;
    }
    if (r.io_type != "binary") stop("io_type = '" + r.io_type + "': only 'binary' dumps are built");
    mkdir(out.c_str(), 0755);

    // init_param + init (init.f90:18-122)
    dg_ctx *ctx = nullptr;
    check(dg_init(&r.p, &ctx), "dg_init");
    std::vector<double> uin((size_t)dg_uin_size(&r.p));
    double time = 0.0, dt = 0.0;
    int ndump = 0;
    if (r.restart > 0) {
        ndump = r.restart;
        check(dg_dump_read(ctx, dump_path(out, ndump).c_str(), &time, &dt), "dg_dump_read");
        ndump++;
    } else {
        check(dg_condinit(&r.p, ic_id(ic), beta, amp, seed, uin.data()), "dg_condinit");
        check(dg_upload(ctx, uin.data()), "dg_upload");
        check(dg_boundary(ctx, 0.0, 0.0), "dg_boundary");
    }
    // the history sums are 3D (history.f90 writes nothing in 2D); the MRI problem has its own
    // routine (src/problem/mri/history.f90), the others use src/subroutines/history.f90
    const bool history_on = r.p.ndim == 3;
    const int hist_variant = ic == "mri" ? DG_HISTORY_MRI : DG_HISTORY_DEFAULT;
    const std::string hist_file = out + "/history.txt";
    auto history = [&]() {
        if (!history_on) return;
        double s[9];
        check(dg_history_variant(ctx, hist_variant, s), "dg_history_variant");
        write_history(hist_file, time, dt, s);
    };
    if (r.restart == 0) {  // dumses.f90:62-67
        check(dg_dump_write(ctx, dump_path(out, ndump).c_str(), time, dt), "dg_dump_write");
        ndump++;
        history();
    }
    double thist = time, tdump = time;
    const long long ncell = (long long)r.p.nx * r.p.ny * r.p.nz;
    const auto t_run0 = std::chrono::steady_clock::now();
    long long step = 0;
    const bool dissipative = r.p.nu > 0.0 || r.p.eta > 0.0;
    for (;;) {  // dumses.f90:75-160
        const auto t0 = std::chrono::steady_clock::now();
        check(dg_compute_dt(ctx, &dt), "dg_compute_dt");
        check(dg_godunov(ctx, dt, time), "dg_godunov");
        if (r.p.fargo) check(dg_fargo_update(ctx, dt), "dg_fargo_update");
        check(dg_boundary(ctx, time, dt), "dg_boundary");
        if (dissipative) check(dg_dissipation(ctx, time, dt), "dg_dissipation");
        if (!quiet) {
            check(dg_sync(ctx), "dg_sync");
            const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            std::printf("Time/dt: %s, %s\n", fortran_1pe(time, 14).c_str(), fortran_1pe(dt, 14).c_str());
            std::printf("Elapsed time, cell update: %.6E s, %.6E cells/s\n", el, (double)ncell / el);
        }
        time = time + dt;
        step++;
        if (r.debug) {  // dumses.f90:123-132
            history();
            thist = thist + r.dthist;
            check(dg_dump_write(ctx, dump_path(out, ndump).c_str(), time, dt), "dg_dump_write");
            ndump++;
            tdump = tdump + r.dtdump;
        } else {
            if ((time - dt) <= (thist + r.dthist) && time > (thist + r.dthist)) {
                history();
                thist = thist + r.dthist;
            }
            if ((time - dt) <= (tdump + r.dtdump) && time > (tdump + r.dtdump)) {
                check(dg_dump_write(ctx, dump_path(out, ndump).c_str(), time, dt), "dg_dump_write");
                ndump++;
                tdump = tdump + r.dtdump;
            }
        }
        if (r.debug ? ndump > 5 : (time - dt) > r.tlim) break;
        if (nsteps >= 0 && step >= nsteps) break;
    }
    check(dg_sync(ctx), "dg_sync");
    const double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_run0).count();
    if (!final_dump.empty()) check(dg_dump_write(ctx, final_dump.c_str(), time, dt), "dg_dump_write");
    std::printf("\n   Elapsed time : %10.3E s\n   Steps        : %lld\n   Zone-cycles/s: %10.3E\n\n", total, step,
                (double)ncell * (double)step / total);
    check(dg_finalize(ctx), "dg_finalize");
    return 0;
}
