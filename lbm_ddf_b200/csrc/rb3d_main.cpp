// rb3d — host driver with the run surface of Summer536/LBM_DDF's single-GPU
// program (src/main.cu), running the B200 engine through the C ABI of
// include/lbm_ddf.h.
//
// Run surface: the fields of src/parameters.h:5-31, read at run time from a
// parameters.h-style file (--params FILE: "#define NAME value" lines, values
// may be arithmetic expressions over earlier names, e.g. BETA
// (0.1 / (LY * 5.0))) and/or from --NAME value options; unset fields take
// the reference's defaults.  Engine choices: --sides wall|periodic (default
// wall, the reference's box), --storage f64|f32|f16s|bf16s (default f64),
// --collision bgk|regularized (default bgk, the reference's), --init
// rest|conduction, --seed, --amplitude, --device.
//
// Behaviour of src/main.cu:11-93: CONTINUE_STEP = 0 starts from the rest
// state of init_arrays (or the seeded conduction state with --init
// conduction); CONTINUE_STEP > 0 reads Ra%.1ePr%.2f/%09d.dat and
// fg%09d.dat (src/initial.cu:110-205).  Steps CONTINUE_STEP+1 .. NEND; every
// NDIAG steps diag_flow (stdout + statistics.dat), every NFLOWOUT steps and
// at NEND output_flow (%09d.dat), every NNUOUT steps output_nu and
// output_profile (Nu_*.txt, Profile_*.txt), at NEND output_fg (fg%09d.dat),
// in the reference's text and binary formats (src/output.cu).  Errors print
// a message and exit with status 1, as the reference does.
#include <sys/stat.h>
#include <sys/time.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <initializer_list>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "lbm_ddf.h"

namespace {

// ---- parameters.h-style values -------------------------------------------

struct Expr {
    // recursive-descent evaluator for numbers, names, + - * / and parentheses
    const std::map<std::string, double> &vars;
    const char *p;
    explicit Expr(const std::map<std::string, double> &v, const char *s) : vars(v), p(s) {}
    void ws() {
        while (*p && std::isspace((unsigned char)*p)) ++p;
    }
    double atom() {
        ws();
        if (*p == '(') {
            ++p;
            double v = sum();
            ws();
            if (*p != ')') throw std::runtime_error("missing )");
            ++p;
            return v;
        }
        if (*p == '-') {
            ++p;
            return -atom();
        }
        if (*p == '+') {
            ++p;
            return atom();
        }
        if (std::isalpha((unsigned char)*p) || *p == '_') {
            std::string name;
            while (std::isalnum((unsigned char)*p) || *p == '_') name += *p++;
            auto it = vars.find(name);
            if (it == vars.end()) throw std::runtime_error("unknown name " + name);
            return it->second;
        }
        char *end = nullptr;
        double v = std::strtod(p, &end);
        if (end == p) throw std::runtime_error(std::string("bad value at '") + p + "'");
        p = end;
        return v;
    }
    double prod() {
        double v = atom();
        for (;;) {
            ws();
            if (*p == '*') { ++p; v *= atom(); }
            else if (*p == '/') { ++p; v /= atom(); }
            else return v;
        }
    }
    double sum() {
        double v = prod();
        for (;;) {
            ws();
            if (*p == '+') { ++p; v += prod(); }
            else if (*p == '-') { ++p; v -= prod(); }
            else return v;
        }
    }
};

struct RunSurface {
    std::map<std::string, double> v;
    std::map<std::string, std::string> raw;   // as written, for expressions
    RunSurface() {
        // defaults of src/parameters.h:5-31
        v["CONTINUE_STEP"] = 0;
        v["LX"] = 400;
        v["LY"] = 400;
        v["LZ"] = 400;
        v["NEND"] = 1000;
        v["NDIAG"] = 10000;
        v["NFLOWOUT"] = 10000;
        v["NNUOUT"] = 10000;
        v["RAYLEIGH"] = 1.0e7;
        v["PRANDTL"] = 0.71;
        v["T_HOT"] = 1.0;
        v["T_COLD"] = 0.0;
        v["GRAVITY"] = 1.0;
        raw["BETA"] = "(0.1 / (LY * 5.0))";
    }
    void set(const std::string &name, const std::string &text) {
        raw[name] = text;
        v.erase(name);
    }
    // evaluates raw expressions once the numeric names they use exist
    void resolve() {
        for (int pass = 0; pass < 8 && !raw.empty(); pass++) {
            for (auto it = raw.begin(); it != raw.end();) {
                try {
                    Expr e(v, it->second.c_str());
                    double x = e.sum();
                    v[it->first] = x;
                    it = raw.erase(it);
                } catch (const std::exception &) {
                    ++it;
                }
            }
        }
        if (!raw.empty()) throw std::runtime_error("cannot evaluate " + raw.begin()->first + " = " + raw.begin()->second);
    }
    double get(const char *k) const { return v.at(k); }
    int geti(const char *k) const { return (int)std::llround(v.at(k)); }
};

void read_params_file(const std::string &path, RunSurface &rs) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error("cannot open " + path);
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        std::string tok, name;
        if (!(ls >> tok) || tok != "#define") continue;
        if (!(ls >> name)) continue;
        std::string rest;
        std::getline(ls, rest);
        auto cpos = rest.find("//");
        if (cpos != std::string::npos) rest = rest.substr(0, cpos);
        while (!rest.empty() && std::isspace((unsigned char)rest.back())) rest.pop_back();
        if (rest.empty()) continue;                          // include guards
        if (name == "LXYZ" || name == "NPOP" || name.rfind("BLOCK_", 0) == 0) continue;
        rs.set(name, rest);
    }
}

void die(const std::string &msg) {
    std::fprintf(stderr, "%s\n", msg.c_str());
    std::exit(EXIT_FAILURE);
}

void check(int rc, const char *what) {
    if (rc != LBM_OK) die(std::string(what) + " failed: " + lbm_last_error());
}

// ---- reference output formats ------------------------------------------------

std::string case_dir(double ra, double pr) {
    char b[256];
    std::snprintf(b, sizeof b, "Ra%.1ePr%.2f", ra, pr);   // src/output.cu:5
    return b;
}

void ensure_dir(const std::string &d) {
    struct stat st;
    if (stat(d.c_str(), &st) == -1) {
        mkdir(d.c_str(), 0700);
        std::printf("Created directory: %s\n", d.c_str());
    }
}

std::string series_name(const std::string &dir, const char *stem, double ra) {
    // src/output.cu:164-178 and :298-312
    char b[512];
    const char *known = nullptr;
    if (ra == 1e5) known = "1e50";
    else if (ra == 5e5) known = "5e50";
    else if (ra == 1e6) known = "1e60";
    else if (ra == 5e6) known = "5e60";
    else if (ra == 1e7) known = "1e70";
    else if (ra == 1e8) known = "1e80";
    if (known) std::snprintf(b, sizeof b, "%s/%s_%s.txt", dir.c_str(), stem, known);
    else std::snprintf(b, sizeof b, "%s/%s_%.2e.txt", dir.c_str(), stem, ra);
    return b;
}

FILE *open_or_die(const std::string &path, const char *mode) {
    FILE *f = std::fopen(path.c_str(), mode);
    if (!f) die("Cannot open file: " + path);
    return f;
}

void write_doubles(FILE *f, const double *a, size_t n, const std::string &what) {
    if (std::fwrite(a, sizeof(double), n, f) != n) die("Error writing " + what);
}

void read_doubles(FILE *f, double *a, size_t n, const std::string &what) {
    if (std::fread(a, sizeof(double), n, f) != n) die("Error reading " + what);
}

struct Driver {
    lbm_params p{};
    lbm_case *c = nullptr;
    size_t N = 0;
    std::string dir;

    void diag_flow(int istep) {   // src/output.cu:3-65
        ensure_dir(dir);
        lbm_observables o;
        check(lbm_get_observables(c, &o, nullptr), "observables");
        std::printf("Step %-7d umean = %14.6e, vmean = %14.6e, wmean = %14.6e, tmean = %14.6e\n", istep, o.ux_mean,
                    o.uy_mean, o.uz_mean, o.phi_mean);
        std::fflush(stdout);
        FILE *f = open_or_die(dir + "/statistics.dat", "a");
        if (std::fprintf(f, "%-7d %14.6e %14.6e %14.6e %14.6e\n", istep, o.ux_mean, o.uy_mean, o.uz_mean,
                         o.phi_mean) < 0)
            die("Error writing to statistics file");
        std::fclose(f);
    }
    void output_flow(int istep) {   // src/output.cu:67-146
        ensure_dir(dir);
        std::vector<double> a(5 * N);
        check(lbm_store_ref_state(c, &a[0], &a[N], &a[2 * N], &a[3 * N], &a[4 * N], nullptr, nullptr), "store");
        char name[512];
        std::snprintf(name, sizeof name, "%s/%09d.dat", dir.c_str(), istep);
        FILE *f = open_or_die(name, "wb");
        write_doubles(f, a.data(), 5 * N, "flow field");
        std::fclose(f);
    }
    void output_nu(int istep) {   // src/output.cu:148-280
        ensure_dir(dir);
        FILE *f = open_or_die(series_name(dir, "Nu", p.rayleigh), "a");
        lbm_observables o;
        check(lbm_get_observables(c, &o, nullptr), "observables");
        if (std::fprintf(f, "%15.6E%15.6E%15.6E%15.6E%15.6E\n", (double)istep, 0.0, o.nu_bulk, o.nu_top,
                         o.nu_bottom) < 0)
            die("Error writing to Nu file");
        std::fclose(f);
    }
    void output_profile(int istep) {   // src/output.cu:282-377
        ensure_dir(dir);
        FILE *f = open_or_die(series_name(dir, "Profile", p.rayleigh), "a");
        std::vector<double> prof(5 * (size_t)p.ly);
        check(lbm_get_profile(c, prof.data(), nullptr), "profile");
        std::fprintf(f, "%d\n", istep);
        for (int iy = 0; iy < p.ly; iy++)
            std::fprintf(f, "%14.6e %14.6e %14.6e %14.6e %14.6e\n", prof[5 * iy], prof[5 * iy + 1], prof[5 * iy + 2],
                         prof[5 * iy + 3], prof[5 * iy + 4]);
        std::fclose(f);
    }
    void output_fg(int istep) {   // src/output.cu:379-419
        std::vector<double> fg(54 * N);
        check(lbm_store_ref_state(c, nullptr, nullptr, nullptr, nullptr, nullptr, &fg[0], &fg[27 * N]), "store");
        char name[512];
        std::snprintf(name, sizeof name, "%s/fg%09d.dat", dir.c_str(), istep);
        FILE *f = open_or_die(name, "wb");
        write_doubles(f, fg.data(), 54 * N, "f and g");
        std::fclose(f);
    }
    void load_restart(int step) {   // src/initial.cu:110-205
        std::vector<double> a(5 * N), fg(54 * N);
        char name[512];
        std::snprintf(name, sizeof name, "%s/%09d.dat", dir.c_str(), step);
        FILE *f = open_or_die(name, "rb");
        read_doubles(f, a.data(), 5 * N, name);
        std::fclose(f);
        std::snprintf(name, sizeof name, "%s/fg%09d.dat", dir.c_str(), step);
        f = open_or_die(name, "rb");
        read_doubles(f, fg.data(), 54 * N, name);
        std::fclose(f);
        check(lbm_load_ref_state(c, &a[0], &a[N], &a[2 * N], &a[3 * N], &a[4 * N], &fg[0], &fg[27 * N]),
              "load restart");
    }
};

void usage() {
    std::printf(
        "usage: rb3d [--params parameters.h] [--NAME value ...] [--sides wall|periodic]\n"
        "            [--storage f64|f32|f16s|bf16s] [--collision bgk|regularized]\n"
        "            [--init rest|conduction] [--seed N] [--amplitude A] [--device D] [--dry-run]\n"
        "NAME is one of CONTINUE_STEP LX LY LZ NEND NDIAG NFLOWOUT NNUOUT RAYLEIGH PRANDTL\n"
        "T_HOT T_COLD GRAVITY BETA (src/parameters.h); values may be expressions.\n");
}

}  // namespace

int main(int argc, char **argv) {
    struct timeval start_time, end_time;
    gettimeofday(&start_time, nullptr);
    RunSurface rs;
    std::string sides = "wall", storage = "f64", init = "rest", collision = "bgk";
    bool dry_run = false;
    unsigned long long seed = 1;
    double amplitude = 1e-3;
    int device = 0;
    try {
        for (int i = 1; i < argc; i++) {
            std::string a = argv[i];
            if (a == "-h" || a == "--help") {
                usage();
                return 0;
            }
            if (a == "--dry-run") {
                dry_run = true;
                continue;
            }
            if (a.rfind("--", 0) != 0 || i + 1 >= argc) {
                usage();
                return 1;
            }
            std::string key = a.substr(2), val = argv[++i];
            if (key == "params") read_params_file(val, rs);
            else if (key == "sides") sides = val;
            else if (key == "storage") storage = val;
            else if (key == "collision") collision = val;
            else if (key == "init") init = val;
            else if (key == "seed") seed = std::strtoull(val.c_str(), nullptr, 10);
            else if (key == "amplitude") amplitude = std::atof(val.c_str());
            else if (key == "device") device = std::atoi(val.c_str());
            else rs.set(key, val);
        }
        rs.resolve();
        if (collision != "bgk" && collision != "regularized")
            throw std::runtime_error("--collision must be bgk or regularized");
    } catch (const std::exception &e) {
        die(std::string("rb3d: ") + e.what());
    }

    Driver d;
    d.p.lx = rs.geti("LX");
    d.p.ly = rs.geti("LY");
    d.p.lz = rs.geti("LZ");
    d.p.sides = sides == "periodic" ? LBM_SIDES_PERIODIC : LBM_SIDES_WALL;
    d.p.storage = storage == "f32" ? LBM_STORE_F32 : storage == "f16s" ? LBM_STORE_F16S
                  : storage == "bf16s" ? LBM_STORE_BF16S : LBM_STORE_F64;
    d.p.device = device;
    d.p.rayleigh = rs.get("RAYLEIGH");
    d.p.prandtl = rs.get("PRANDTL");
    d.p.t_hot = rs.get("T_HOT");
    d.p.t_cold = rs.get("T_COLD");
    d.p.gravity = rs.get("GRAVITY");
    d.p.beta = rs.get("BETA");
    const int nend = rs.geti("NEND"), ndiag = rs.geti("NDIAG"), nflow = rs.geti("NFLOWOUT"),
              nnu = rs.geti("NNUOUT"), cont = rs.geti("CONTINUE_STEP");
    if (ndiag <= 0 || nflow <= 0 || nnu <= 0) die("rb3d: output intervals must be positive");
    d.N = (size_t)d.p.lx * d.p.ly * d.p.lz;
    d.dir = case_dir(d.p.rayleigh, d.p.prandtl);
    if (dry_run) {   // resolved run surface and derived parameters, no GPU needed
        lbm_derived dv;
        check(lbm_derive(&d.p, &dv), "lbm_derive");
        for (const auto &kv : rs.v) std::printf("%s = %.17g\n", kv.first.c_str(), kv.second);
        std::printf("visc = %.17g\ntau = %.17g\nu0 = %.17g\ndiff = %.17g\ntauc = %.17g\nt0 = %.17g\n", dv.visc,
                    dv.tau, dv.u0, dv.diff, dv.tauc, dv.t0);
        std::printf("dir = %s\n", d.dir.c_str());
        return 0;
    }

    check(lbm_create(&d.p, &d.c), "lbm_create");
    check(lbm_set_collision(d.c, collision == "regularized" ? LBM_COLLISION_REGULARIZED : LBM_COLLISION_BGK),
          "lbm_set_collision");
    if (cont == 0) {
        if (init == "conduction") check(lbm_init_conduction(d.c, seed, amplitude, nullptr), "init");
        else check(lbm_init_rest(d.c, nullptr), "init");
    } else {
        d.load_restart(cont);
    }

    double gpu_time = 0.0, cpu_time = 0.0;
    // steps between output events run back to back; events timed as the
    // reference's "GPU computation time" (src/main.cu:25-56)
    int istep = cont;
    while (istep < nend) {
        int next = nend;
        for (int every : {ndiag, nflow, nnu}) next = std::min(next, (istep / every + 1) * every);
        const int n = next - istep;
        struct timeval t0, t1;
        gettimeofday(&t0, nullptr);
        check(lbm_step(d.c, n, nullptr), "lbm_step");
        lbm_observables o;
        int rc = lbm_get_observables(d.c, &o, nullptr);   // also synchronises
        gettimeofday(&t1, nullptr);
        gpu_time += (t1.tv_sec - t0.tv_sec) + (t1.tv_usec - t0.tv_usec) / 1e6;
        if (rc == LBM_ERR_DIVERGED) std::fprintf(stderr, "warning: NaN/Inf in the fields at step %d\n", next);
        else check(rc, "observables");
        istep = next;
        clock_t cs = std::clock();
        if (istep % ndiag == 0) d.diag_flow(istep);
        if (istep % nflow == 0 || istep == nend) d.output_flow(istep);
        if (istep % nnu == 0) {
            d.output_nu(istep);
            d.output_profile(istep);
        }
        if (istep == nend) d.output_fg(istep);
        cpu_time += (double)(std::clock() - cs) / CLOCKS_PER_SEC;
    }
    gettimeofday(&end_time, nullptr);
    const double total = (end_time.tv_sec - start_time.tv_sec) + (end_time.tv_usec - start_time.tv_usec) / 1e6;
    std::printf("Simulation completed.\n");
    std::printf("Rayleigh number: %.2e\n", d.p.rayleigh);
    std::printf("Prandtl number: %.2f\n", d.p.prandtl);
    std::printf("Total iterations: %d\n", nend);
    std::printf("CPU computation time: %.2f seconds\n", cpu_time);
    std::printf("GPU computation time: %.2f seconds\n", gpu_time);
    std::printf("Total computation time: %.2f seconds\n", total);
    if (gpu_time > 0) std::printf("MLUPS: %.1f\n", (double)d.N * (nend - cont) / gpu_time / 1e6);
    lbm_destroy(d.c);
    return 0;
}
