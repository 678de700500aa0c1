// driver.cpp -- cavity_les: the reference binary (src/main.rs, src/cli.rs)
// over the C ABI of libcavity_b200.so.
//
//   command line   parse_args (src/cli.rs:185-384): the same flags, aliases,
//                  defaults, checks and exit codes; --precision, --device
//                  and --geq-order are additions (storage format, CUDA
//                  device, form of the g equilibrium);
//   run_uniform    src/main.rs:42-443;
//   run_octree     src/main.rs:447-720.
//
// The step loop runs on the GPU in chunks between the driver's events
// (progress line + guards every --progress-every steps, a time-average
// sample every --sample-every steps from --sample-start, a snapshot every
// --snapshot-every steps): each chunk is one cav_step call (CUDA graphs
// inside), the diagnostics are device reductions, the time average stays on
// the device.  Fields cross to the host only for snapshots, the divergence
// report and the final exports.  Text outputs use Rust's float formats
// (rustfmt.h), so FP64 runs write the reference's bytes for its values.
#include <sys/stat.h>

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <string>
#include <thread>
#include <vector>

#include "cavity.h"
#include "rustfmt.h"

namespace {

constexpr double MAX_U_ABORT = 0.10;   // src/main.rs:46, src/octree/cavity.rs:42
constexpr double DELTA_T = 1.0;        // T_HOT - T_COLD (src/uniform/solver.rs:21)
constexpr double OCT_UTARGET = 0.02;   // src/octree/cavity.rs:45

enum class Mode { Uniform, Octree };

// Args::default, src/cli.rs:94-130.
struct Args {
    Mode mode = Mode::Uniform;
    long long nx = 64, ny = 256;
    double ra = 1.0e6, pr = 0.71, cs = 0.10, pr_t = 0.9;
    long long steps = 200000, sample_start = 100000, sample_every = 100;
    std::string out = "output/runs_uniforme/ra1e6";
    double utarget = 0.02;
    unsigned long long seed = 42;
    long long progress_every = 1000, jobs = 1;
    double alpha_mult = 1.0, nu_start_mult = 1.0;
    bool has_restart = false;
    std::string restart;
    bool has_nu = false;
    double nu = 0.0;
    long long snapshot_every = 0;
    bool dynamic_smag = false;
    double smag_alpha = 0.5, nu_sm_min = -0.1, eta_test = 2.0;
    long long nx0 = 64, ny0 = 256, bl_width = 8;
    bool odd_exact = false;
    long long levels = 2;
    // additions of this build
    std::string precision = "f64";
    int device = 0;
    int geq_order = 2;
};

const char* USAGE =
    "Usage: cavity_les [OPTIONS]\n"
    "\n"
    "Differentially heated cavity (D2Q9 TRT lattice Boltzmann, Smagorinsky LES) on the GPU.\n"
    "\n"
    "  --mode <uniform|octree>   uniform grid (default) or block-refined octree\n"
    "\n"
    "Uniform grid:\n"
    "  --nx <n> / --ny <n>       grid width / height             [64 / 256]\n"
    "  --cs <f> / --pr_t <f>     Smagorinsky constant / turbulent Prandtl [0.1 / 0.9]\n"
    "  --alpha-mult <f>          thermal diffusivity multiplier   [1.0]\n"
    "\n"
    "Octree:\n"
    "  --nx0 <n> / --ny0 <n>     coarse grid                      [64 / 256]\n"
    "  --bl-width <n>            fine block width in coarse cells [8]\n"
    "  --levels <2|3>            refinement levels                [2]\n"
    "  --odd-exact               xi_odd from tau- ratio (default 1/2)\n"
    "\n"
    "Both modes:\n"
    "  --ra <f> / --pr <f>       Rayleigh / Prandtl               [1e6 / 0.71]\n"
    "  --steps <n>               time steps (coarse steps)        [200000]\n"
    "  --sample-start <n>        first averaged step              [100000]\n"
    "  --sample-every <n>        averaging stride                 [100]\n"
    "  --progress-every <n>      progress line period             [1000]\n"
    "  --out <dir>               output directory                 [output/runs_uniforme/ra1e6]\n"
    "  --utarget <f>             velocity target of the nu calibration [0.02]\n"
    "  --seed <n>                initial-noise seed               [42]\n"
    "  --jobs <n>                accepted; the GPU ignores it     [1]\n"
    "  --nu-start-mult <f>       initial viscosity multiplier     [1.0]\n"
    "  --nu <f>                  forced viscosity (< 0.002)\n"
    "  --restart <file>          start from a snapshot (CAVSNAP1 / OCTSNAP1)\n"
    "  --snapshot-every <n>      rewrite snapshot.bin every n steps [0 = off]\n"
    "  --dynamic-smag            dynamic mixed-scale subgrid model\n"
    "  --smag-alpha <f>          mixed-form exponent              [0.5]\n"
    "  --nu-sm-min <f>           lower bound nu_sm >= nu_sm_min nu [-0.1]\n"
    "  --eta-test <f>            test-filter ratio                [2.0]\n"
    "\n"
    "GPU:\n"
    "  --precision <p>           uniform: f64 f32 f16 bf16 f16g f16sr bf16sr f16gsr;\n"
    "                            octree: f64 f32 f32_f16 f32_f16g  [f64]\n"
    "  --device <n>              CUDA device ordinal              [0]\n"
    "  --geq-order <1|2>         uniform: g equilibrium linear / quadratic in u [2]\n";

struct ArgError {
    std::string msg;
};

bool parse_u(const std::string& v, long long& out) {
    if (v.empty() || v[0] == '-' || v[0] == '+') return false;
    char* end = nullptr;
    errno = 0;
    const unsigned long long x = std::strtoull(v.c_str(), &end, 10);
    if (errno || *end || x > (unsigned long long)INT64_MAX) return false;
    out = (long long)x;
    return true;
}
bool parse_u64(const std::string& v, unsigned long long& out) {
    if (v.empty() || v[0] == '-' || v[0] == '+') return false;
    char* end = nullptr;
    errno = 0;
    out = std::strtoull(v.c_str(), &end, 10);
    return !errno && !*end;
}
bool parse_f(const std::string& v, double& out) {
    if (v.empty() || std::isspace((unsigned char)v[0])) return false;
    char* end = nullptr;
    out = std::strtod(v.c_str(), &end);
    return *end == '\0';
}

// parse_args, src/cli.rs:188-384.
Args parse_args(int argc, char** argv, bool& help) {
    Args a;
    help = false;
    std::vector<std::string> av(argv + 1, argv + argc);
    for (size_t i = 0; i < av.size(); ++i) {
        const std::string& arg = av[i];
        const size_t eq = arg.find('=');
        std::string key = arg.substr(0, eq);
        key.erase(0, key.find_first_not_of('-') == std::string::npos ? key.size() : key.find_first_not_of('-'));
        const bool has_inline = eq != std::string::npos;
        const std::string inline_val = has_inline ? arg.substr(eq + 1) : "";
        auto boolean = [&](bool& dst, const char* name) {
            if (!has_inline) dst = true;
            else if (inline_val == "true" || inline_val == "1") dst = true;
            else if (inline_val == "false" || inline_val == "0") dst = false;
            else throw ArgError{std::string("--") + name + ": boolean expected, got '" + inline_val + "'"};
        };
        if (key == "dynamic-smag" || key == "dynamic_smag") {
            boolean(a.dynamic_smag, "dynamic-smag");
            continue;
        }
        if (key == "odd-exact" || key == "odd_exact") {
            boolean(a.odd_exact, "odd-exact");
            continue;
        }
        if (key == "help" || key == "h") {
            help = true;
            return a;
        }
        std::string value;
        if (has_inline) {
            value = inline_val;
        } else {
            if (i + 1 >= av.size()) throw ArgError{"missing value for --" + key};
            value = av[++i];
        }
        auto uint_of = [&](long long& dst, const char* name) {
            if (!parse_u(value, dst)) throw ArgError{std::string("--") + name + ": integer expected, got '" + value + "'"};
        };
        auto float_of = [&](double& dst, const char* name) {
            if (!parse_f(value, dst)) throw ArgError{std::string("--") + name + ": number expected, got '" + value + "'"};
        };
        if (key == "mode") {
            std::string m = value;
            std::transform(m.begin(), m.end(), m.begin(), ::tolower);
            if (m == "uniform") a.mode = Mode::Uniform;
            else if (m == "octree") a.mode = Mode::Octree;
            else throw ArgError{"--mode: 'uniform' or 'octree' expected, got '" + m + "'"};
        } else if (key == "nx") uint_of(a.nx, "nx");
        else if (key == "ny") uint_of(a.ny, "ny");
        else if (key == "ra") float_of(a.ra, "ra");
        else if (key == "pr") float_of(a.pr, "pr");
        else if (key == "cs") float_of(a.cs, "cs");
        else if (key == "pr_t" || key == "prt") float_of(a.pr_t, "pr_t");
        else if (key == "steps") uint_of(a.steps, "steps");
        else if (key == "sample-start" || key == "sample_start") uint_of(a.sample_start, "sample-start");
        else if (key == "sample-every" || key == "sample_every") uint_of(a.sample_every, "sample-every");
        else if (key == "out") a.out = value;
        else if (key == "utarget") float_of(a.utarget, "utarget");
        else if (key == "seed") {
            if (!parse_u64(value, a.seed)) throw ArgError{"--seed: integer expected, got '" + value + "'"};
        } else if (key == "progress-every" || key == "progress_every") uint_of(a.progress_every, "progress-every");
        else if (key == "jobs" || key == "j") uint_of(a.jobs, "jobs");
        else if (key == "alpha-mult" || key == "alpha_mult") float_of(a.alpha_mult, "alpha-mult");
        else if (key == "nu-start-mult" || key == "nu_start_mult") float_of(a.nu_start_mult, "nu-start-mult");
        else if (key == "restart") {
            a.has_restart = true;
            a.restart = value;
        } else if (key == "smag-alpha" || key == "smag_alpha") float_of(a.smag_alpha, "smag-alpha");
        else if (key == "nu-sm-min" || key == "nu_sm_min") float_of(a.nu_sm_min, "nu-sm-min");
        else if (key == "eta-test" || key == "eta_test") float_of(a.eta_test, "eta-test");
        else if (key == "snapshot-every" || key == "snapshot_every") uint_of(a.snapshot_every, "snapshot-every");
        else if (key == "nu") {
            double v;
            float_of(v, "nu");
            if (!(v > 0.0) || !std::isfinite(v)) throw ArgError{"--nu must be > 0 and finite"};
            if (v >= 0.002)
                throw ArgError{"--nu " + rf::display(v) +
                               " >= 0.002: the utarget calibration covers it; --nu is for values below the 0.002 floor"};
            a.has_nu = true;
            a.nu = v;
        } else if (key == "nx0") uint_of(a.nx0, "nx0");
        else if (key == "ny0") uint_of(a.ny0, "ny0");
        else if (key == "bl-width" || key == "bl_width") uint_of(a.bl_width, "bl-width");
        else if (key == "levels") uint_of(a.levels, "levels");
        else if (key == "precision") a.precision = value;
        else if (key == "geq-order" || key == "geq_order") {
            long long o;
            uint_of(o, "geq-order");
            if (o != 1 && o != 2) throw ArgError{"--geq-order: 1 or 2 expected"};
            a.geq_order = int(o);
        }
        else if (key == "device") {
            long long d;
            uint_of(d, "device");
            a.device = int(d);
        } else throw ArgError{"unknown option '--" + key + "'"};
    }
    if (a.nx < 8 || a.ny < 8) throw ArgError{"nx and ny must be >= 8"};
    if (a.ny <= a.nx) throw ArgError{"tall cavity: ny must be > nx (Az ~ 4)"};
    if (a.ra <= 0.0 || a.pr <= 0.0) throw ArgError{"ra and pr must be > 0"};
    if (a.sample_every == 0) throw ArgError{"sample-every must be >= 1"};
    if (a.jobs == 0) throw ArgError{"jobs must be >= 1"};
    if (!(a.alpha_mult > 0.0) || !std::isfinite(a.alpha_mult)) throw ArgError{"alpha-mult must be > 0 and finite"};
    if (!(a.nu_start_mult >= 1.0) || !std::isfinite(a.nu_start_mult))
        throw ArgError{"nu-start-mult must be >= 1 and finite"};
    if (!(a.smag_alpha >= 0.0 && a.smag_alpha <= 1.0) || !std::isfinite(a.smag_alpha))
        throw ArgError{"smag-alpha must be in [0, 1] (0 = pure Smagorinsky, 1 = pure similarity)"};
    if (!(a.eta_test >= 1.0) || !std::isfinite(a.eta_test)) throw ArgError{"eta-test must be >= 1"};
    if (a.mode == Mode::Octree) {
        if (a.nx0 < 16 || a.ny0 < 16) throw ArgError{"nx0 and ny0 must be >= 16"};
        if (a.ny0 <= a.nx0) throw ArgError{"tall cavity: ny0 must be > nx0 (Az ~ 4)"};
        if (!(a.bl_width >= 2 && 2 * a.bl_width < a.nx0))
            throw ArgError{"bl-width must be >= 2 and 2 bl-width < nx0 (a coarse core is required)"};
        if (!(a.levels == 2 || a.levels == 3)) throw ArgError{"levels must be 2 or 3"};
        if (a.levels == 3 && a.bl_width != 4)
            std::fprintf(stderr, "Note : escalier V6 conçu pour bl-width = 4 cellules grossières (frontières tanh §0.1) ; lu %lld\n",
                         a.bl_width);
    }
    // progress_every = 0 is a division by zero in the reference's loop
    if (a.progress_every == 0) throw ArgError{"progress-every must be >= 1"};
    return a;
}

// ---- small helpers ----------------------------------------------------------
void out_line(const std::string& s) {
    std::fwrite(s.data(), 1, s.size(), stdout);
    std::fputc('\n', stdout);
    std::fflush(stdout);
}
void err_line(const std::string& s) {
    std::fwrite(s.data(), 1, s.size(), stderr);
    std::fputc('\n', stderr);
}

bool create_dir_all(const std::string& path, std::string& err) {
    std::string cur;
    for (size_t i = 0; i <= path.size(); ++i) {
        if (i == path.size() || path[i] == '/') {
            cur = path.substr(0, i);
            if (!cur.empty() && ::mkdir(cur.c_str(), 0777) != 0 && errno != EEXIST) {
                err = std::strerror(errno);
                return false;
            }
        }
    }
    struct stat st;
    if (::stat(path.c_str(), &st) != 0 || !S_ISDIR(st.st_mode)) {
        err = "not a directory";
        return false;
    }
    return true;
}

std::string join(const std::string& dir, const char* name) {
    if (dir.empty() || dir.back() == '/') return dir + name;
    return dir + "/" + name;
}

bool write_text(const std::string& path, const std::string& text, std::string& err) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) {
        err = std::strerror(errno);
        return false;
    }
    const bool ok = std::fwrite(text.data(), 1, text.size(), f) == text.size();
    if (std::fclose(f) != 0 || !ok) {
        err = "write failed";
        return false;
    }
    return true;
}

// write_log, src/uniform/post.rs:371-376: every line + '\n'.
std::string log_text(const std::vector<std::string>& lines) {
    std::string s;
    for (const std::string& l : lines) s += l + "\n";
    return s;
}

[[noreturn]] void die_cav(const char* what, int rc, const char* msg) {
    err_line(std::string(what) + " failed (" + std::to_string(rc) + "): " + (msg ? msg : ""));
    std::exit(101);
}

// nusselt_trias_2d, src/uniform/post.rs:327-346: log-log interpolation
// between the anchors, the power-law fit outside.
double nusselt_trias_2d(double ra) {
    const double A[3][2] = {{6.4e8, 49.23}, {2e9, 66.19}, {1e10, 100.60}};
    if (ra <= A[0][0] || ra >= A[2][0]) return 0.2529 * std::pow(ra, 0.26);
    for (int w = 0; w < 2; ++w) {
        const double ra_i = A[w][0], nu_i = A[w][1], ra_j = A[w + 1][0], nu_j = A[w + 1][1];
        if (ra >= ra_i && ra <= ra_j) {
            const double t = (std::log(ra) - std::log(ra_i)) / (std::log(ra_j) - std::log(ra_i));
            return std::exp(std::log(nu_i) + t * (std::log(nu_j) - std::log(nu_i)));
        }
    }
    return 0.0;
}

// max_of / max_of_range, src/main.rs:757-784.
void max_of_range(const std::vector<double>& p, size_t i0, size_t i1, size_t nx, double& best, double& x) {
    best = 0.0;
    size_t bi = i0;
    for (size_t i = i0; i < i1 && i < p.size(); ++i)
        if (std::fabs(p[i]) > best) {
            best = std::fabs(p[i]);
            bi = i;
        }
    x = double(bi) / double(nx - 1);
}
void max_of(const std::vector<double>& p, size_t nx, double& best, double& x) {
    best = 0.0;
    size_t bi = 1;
    for (size_t i = 1; i < 1 + (nx >= 2 ? nx - 2 : 0) && i < p.size(); ++i)
        if (std::fabs(p[i]) > best) {
            best = std::fabs(p[i]);
            bi = i;
        }
    x = double(bi) / double(nx - 1);
}

// Next step index >= s at which the loop must stop for an event.
long long next_event(long long s, long long steps, long long pe, long long ss, long long se, long long sn,
                     bool sample_events) {
    long long e = steps - 1;
    e = std::min(e, ((s + pe - 1) / pe) * pe);
    if (sample_events && ss < steps) e = std::min(e, s <= ss ? ss : ss + ((s - ss + se - 1) / se) * se);
    if (sn > 0) e = std::min(e, ((s + sn) / sn) * sn - 1);
    return std::max(e, s);
}

int uniform_precision(const std::string& p) {
    const char* names[] = {"f64", "f32", "f16", "bf16", "f16g", "f16sr", "bf16sr", "f16gsr"};
    for (int i = 0; i < 8; ++i)
        if (p == names[i]) return i;
    return -1;
}
int octree_precision(const std::string& p) {
    const char* names[] = {"f64", "f32", "f32_f16", "f32_f16g"};
    for (int i = 0; i < 4; ++i)
        if (p == names[i]) return i;
    return -1;
}

// ---- run_uniform, src/main.rs:42-443 -----------------------------------------
int run_uniform(const Args& args) {
    out_line("=== Cavité différentiellement chauffée 2D (LBM D2Q9 + Smagorinsky) ===");
    out_line("Grille : " + std::to_string(args.nx) + "×" + std::to_string(args.ny) + " (Az = " +
             rf::fixed(double(args.ny - 1) / double(args.nx - 1), 2) + ") | Ra = " + rf::exp(args.ra, 3) +
             " | Pr = " + rf::display(args.pr) + " | Cs = " + rf::display(args.cs) + " | Pr_t = " +
             rf::display(args.pr_t) + " | jobs = " + std::to_string(args.jobs));
    if (args.jobs > 1) {
        const long long cores = std::max(1u, std::thread::hardware_concurrency());
        if (args.jobs > cores)
            err_line("Warning : --jobs " + std::to_string(args.jobs) + " > " + std::to_string(cores) +
                     " cœurs disponibles ; cap à " + std::to_string(cores) + ".");
    }
    const int prec = uniform_precision(args.precision);
    if (prec < 0) {
        err_line("Error: unknown --precision '" + args.precision + "' for the uniform solver");
        return 1;
    }
    cav_params p;
    cav_default_params(&p);
    p.nx = int32_t(args.nx);
    p.ny = int32_t(args.ny);
    p.ra = args.ra;
    p.pr = args.pr;
    p.cs = args.cs;
    p.pr_t = args.pr_t;
    p.utarget = args.utarget;
    p.seed = args.seed;
    p.jobs = int32_t(args.jobs);
    p.alpha_mult = args.alpha_mult;
    p.nu_start_mult = args.nu_start_mult;
    p.has_nu_override = args.has_nu ? 1 : 0;
    p.nu_override = args.nu;
    p.init_mode = CAV_INIT_LINEAR;
    p.noise_amp = 1.0e-3;
    p.geq_order = args.geq_order;
    p.precision = prec;
    p.device = args.device;
    cav_handle* h = nullptr;
    int rc = cav_create(&p, &h);
    if (rc != CAV_OK) die_cav("cav_create", rc, cav_last_error(nullptr));
    auto ck = [&](int r, const char* what) {
        if (r != CAV_OK) die_cav(what, r, cav_last_error(h));
    };
    ck(cav_set_dynamic_sgs(h, args.dynamic_smag ? 1 : 0, args.smag_alpha, args.nu_sm_min, args.eta_test),
       "cav_set_dynamic_sgs");
    if (args.dynamic_smag)
        out_line("LES dynamique : échelles mixtes α = " + rf::display(args.smag_alpha) + " (Tab. 2.3) | η_test = " +
                 rf::display(args.eta_test) + " | νsm_min = " + rf::display(args.nu_sm_min) + "·ν");
    if (args.has_restart) {
        int64_t snx = 0, sny = 0;
        if (cav_snapshot_read_fields(args.restart.c_str(), &snx, &sny, nullptr, nullptr, nullptr, nullptr) != CAV_OK) {
            err_line("Erreur de lecture du snapshot " + args.restart + " : " + cav_last_error(nullptr));
            return 6;
        }
        out_line("Restart depuis " + args.restart + " : snapshot " + std::to_string(snx) + "×" + std::to_string(sny) +
                 " → grille " + std::to_string(args.nx) + "×" + std::to_string(args.ny) +
                 ((snx == args.nx && sny == args.ny) ? "" : " (interpolation bilinéaire)"));
        if (cav_restart_from_snapshot(h, args.restart.c_str()) != CAV_OK) {
            err_line("Erreur de lecture du snapshot " + args.restart + " : " + cav_last_error(h));
            return 6;
        }
    }
    cav_info info;
    ck(cav_get_info(h, &info), "cav_get_info");
    out_line("Unités réseau : nu = " + rf::fixed(info.nu, 6) + " | alpha = " + rf::fixed(info.alpha, 6) +
             " | tau = " + rf::fixed(info.tau, 4) + " | tau_t = " + rf::fixed(info.tau_t, 4) +
             " | beta_eff = " + rf::exp(info.beta_eff, 4));
    const double ra_check = 1.0 * info.beta_eff * DELTA_T * info.lz * info.lz * info.lz / (info.nu * info.alpha_phys);
    out_line("Ra vérifié depuis unités réseau : " + rf::exp(ra_check, 4) + " (cible " + rf::exp(args.ra, 4) + ")");

    const long long nx = args.nx, ny = args.ny, n_nodes = nx * ny;
    std::vector<std::string> log_lines;
    const auto t0 = std::chrono::steady_clock::now();
    std::string snap_path;
    if (args.snapshot_every > 0) {
        std::string e;
        if (!create_dir_all(args.out, e)) {
            err_line("Impossible de créer " + args.out + " : " + e);
            return 4;
        }
        snap_path = join(args.out, "snapshot.bin");
    }
    long long n_samples = 0;
    for (long long s = 0; s < args.steps;) {
        const long long step = next_event(s, args.steps, args.progress_every, args.sample_start, args.sample_every,
                                          args.snapshot_every, true);
        ck(cav_step(h, step - s + 1), "cav_step");
        s = step + 1;
        if (step % args.progress_every == 0 || step + 1 == args.steps) {
            cav_diag_out d;
            ck(cav_diag(h, &d), "cav_diag");
            std::string dyn;
            if (args.dynamic_smag) {
                double st[4];
                ck(cav_dynamic_sgs_stats(h, st), "cav_dynamic_sgs_stats");
                dyn = " | cs_dyn_mean = " + rf::fixed(st[0], 4) + " | cs_dyn_max = " + rf::fixed(st[1], 4) +
                      " | kap_dyn_mean = " + rf::fixed(st[2], 4);
            }
            const std::string msg = "step " + rf::right(std::to_string(step), 7) + " | w_max = " +
                                    rf::fixed(d.max_uy, 5) + " | max_u = " + rf::fixed(d.max_u, 5) + " | Nuc = " +
                                    rf::fixed(d.nusselt_hot, 4) + " | Nuf = " + rf::fixed(d.nusselt_cold, 4) +
                                    " | masse = " + rf::fixed(d.total_mass / double(n_nodes), 6) +
                                    " | nu_t_max = " + rf::exp(d.nu_t_max, 3) + dyn;
            out_line(msg);
            log_lines.push_back(msg);
            if (d.max_u > MAX_U_ABORT) {
                const double ma_local = d.max_u * std::sqrt(3.0);
                const std::string abort_msg = "AVORT : max_u = " + rf::fixed(d.max_u, 5) + " dépasse le garde-fou " +
                                              rf::fixed(MAX_U_ABORT, 2) + " (Ma_local = max_u·√3 ≈ " +
                                              rf::fixed(ma_local, 3) + " > marge de sécurité)";
                err_line(abort_msg);
                log_lines.push_back(abort_msg);
                std::string e;
                create_dir_all(args.out, e);
                write_text(join(args.out, "progress.log"), log_text(log_lines), e);
                return 2;
            }
            if (!d.finite) {
                // the first non-finite field and the population extremes
                // (src/main.rs:230-275)
                std::vector<double> T(n_nodes), U(n_nodes), V(n_nodes), R(n_nodes), F(n_nodes * 9), G(n_nodes * 9);
                ck(cav_get_fields(h, R.data(), U.data(), V.data(), T.data(), nullptr, nullptr), "cav_get_fields");
                ck(cav_get_populations(h, F.data(), G.data()), "cav_get_populations");
                auto first_nf = [](const std::vector<double>& v) -> long long {
                    for (size_t k = 0; k < v.size(); ++k)
                        if (!std::isfinite(v[k])) return (long long)k;
                    return -1;
                };
                auto absmax = [](const std::vector<double>& v, bool& nan) {
                    double m = 0.0;
                    nan = false;
                    for (double x : v) {
                        m = std::fmax(m, std::fabs(x));
                        nan = nan || !std::isfinite(x);
                    }
                    return m;
                };
                bool f_nan, g_nan;
                const double f_max = absmax(F, f_nan), g_max = absmax(G, g_nan);
                const std::pair<const char*, long long> cand[4] = {
                    {"temperature", first_nf(T)}, {"ux", first_nf(U)}, {"uy", first_nf(V)}, {"rho", first_nf(R)}};
                for (const auto& c : cand)
                    if (c.second >= 0) {
                        const long long k = c.second, x = k % nx, y = k / nx;
                        err_line(std::string("DIAG: premier champ non fini = ") + c.first + " au nœud k=" +
                                 std::to_string(k) + " (x=" + std::to_string(x) + ", y=" + std::to_string(y) + "/" +
                                 std::to_string(ny) + ") ; f: max|f|=" + rf::exp(f_max, 6) +
                                 " NaN=" + (f_nan ? "true" : "false") + " ; g: max|g|=" + rf::exp(g_max, 6) +
                                 " NaN=" + (g_nan ? "true" : "false") +
                                 " ; bords: y_proche_paroi=" + std::to_string(std::min(y, ny - 1 - y)));
                        break;
                    }
                err_line("DIVERGENCE détectée au pas " + std::to_string(step) + " (valeurs non finies).");
                return 2;
            }
        }
        if (step >= args.sample_start && (step - args.sample_start) % args.sample_every == 0) {
            ck(cav_sample(h), "cav_sample");
            ++n_samples;
        }
        if (args.snapshot_every > 0 && (step + 1) % args.snapshot_every == 0) {
            if (cav_snapshot_write(h, snap_path.c_str()) != CAV_OK) {
                err_line("Erreur d'export du snapshot au pas " + std::to_string(step) + " : " + cav_last_error(h));
                return 5;
            }
            out_line("snapshot exporté au pas " + std::to_string(step));
        }
    }
    ck(cav_sync(h), "cav_sync");
    const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    out_line("Simulation terminée en " + rf::fixed(elapsed, 1) + " s (" +
             rf::fixed(double(args.steps) / elapsed / 1000.0, 1) + "k pas/s)");
    if (n_samples == 0) {
        err_line("Aucun échantillon moyenné : sample_start ≥ steps ?");
        return 3;
    }
    out_line("Moyennage sur " + std::to_string(n_samples) + " échantillons.");

    // ---- post-processing of the mean fields (src/main.rs:314-344) ----
    const size_t n = size_t(n_nodes);
    std::vector<double> ux_m(n), uy_m(n), t_m(n), nut_m(n), uu_m(n);
    int64_t got = 0;
    ck(cav_get_means(h, ux_m.data(), uy_m.data(), t_m.data(), nut_m.data(), uu_m.data(), &got), "cav_get_means");
    // stream_function_mean (:723-738)
    std::vector<double> psi(n, 0.0);
    for (long long ix = 0; ix < nx; ++ix) {
        double acc = 0.0;
        for (long long iy = 1; iy < ny; ++iy) {
            acc += 0.5 * (ux_m[(iy - 1) * nx + ix] + ux_m[iy * nx + ix]);
            psi[iy * nx + ix] = acc;
        }
    }
    // nusselt_from_mean (:741-754)
    auto nu_mean = [&](bool hot) {
        double sum = 0.0;
        for (long long iy = 0; iy < ny; ++iy) {
            const double grad = hot ? t_m[iy * nx + 1] - t_m[iy * nx + 2] : t_m[iy * nx + nx - 3] - t_m[iy * nx + nx - 2];
            sum += std::fabs(grad);
        }
        return (sum / double(ny)) * info.lz / DELTA_T;
    };
    const double nuc = nu_mean(true), nuf = nu_mean(false);
    const long long iy_mid = ny / 2, iy_075 = 3 * ny / 4;
    std::vector<double> uy_mid(nx), uy_075(nx);
    for (long long ix = 0; ix < nx; ++ix) {
        uy_mid[ix] = uy_m[iy_mid * nx + ix];
        uy_075[ix] = uy_m[iy_075 * nx + ix];
    }
    double wmax_mid, x_mid, wmax_075, x_075, wmax_mid_hot, x_mid_hot, wmax_075_hot, x_075_hot;
    max_of(uy_mid, size_t(nx), wmax_mid, x_mid);
    max_of(uy_075, size_t(nx), wmax_075, x_075);
    max_of_range(uy_mid, 1, size_t(nx / 2), size_t(nx), wmax_mid_hot, x_mid_hot);
    max_of_range(uy_075, 1, size_t(nx / 2), size_t(nx), wmax_075_hot, x_075_hot);
    cav_diag_out fin;
    ck(cav_diag(h, &fin), "cav_diag");
    const double yplus = fin.y_plus_hot;
    double s2 = 0.0;
    for (size_t k = 0; k < n; ++k) s2 += std::fmax(uu_m[k] - ux_m[k] * ux_m[k] - uy_m[k] * uy_m[k], 0.0);
    const double s_half = std::sqrt(s2 / double(n));

    // ---- exports (:346-391) ----
    {
        std::string e;
        if (!create_dir_all(args.out, e)) {
            err_line("Impossible de créer " + args.out + " : " + e);
            return 4;
        }
    }
    std::vector<double> R(n), U(n), V(n), T(n);
    ck(cav_get_fields(h, R.data(), U.data(), V.data(), T.data(), nullptr, nullptr), "cav_get_fields");
    std::string errs[6];
    bool oks[6];
    {  // write_fields_csv (post.rs:201-229)
        std::string s = "x,y,ux,uy,T,psi,nu_t\n";
        s.reserve(n * 96);
        for (long long iy = 0; iy < ny; ++iy)
            for (long long ix = 0; ix < nx; ++ix) {
                const size_t k = size_t(iy * nx + ix);
                s += rf::fixed(double(ix), 6) + "," + rf::fixed(double(iy), 6) + "," + rf::exp(ux_m[k], 8) + "," +
                     rf::exp(uy_m[k], 8) + "," + rf::exp(t_m[k], 8) + "," + rf::exp(psi[k], 8) + "," +
                     rf::exp(nut_m[k], 8) + "\n";
            }
        oks[0] = write_text(join(args.out, "fields_mean.csv"), s, errs[0]);
    }
    {  // write_profiles_csv (:232-247)
        std::string s = "x_norm,w_z05,w_z075\n";
        for (long long ix = 0; ix < nx; ++ix)
            s += rf::fixed(double(ix) / double(nx - 1), 6) + "," + rf::exp(uy_mid[ix], 8) + "," +
                 rf::exp(uy_075[ix], 8) + "\n";
        oks[1] = write_text(join(args.out, "profiles_w.csv"), s, errs[1]);
    }
    {  // write_vtk (:250-303)
        std::string st, su, sv;
        for (long long iy = 0; iy < ny; ++iy) {
            for (long long ix = 0; ix < nx; ++ix) {
                const size_t k = size_t(iy * nx + ix);
                st += rf::exp(T[k], 6) + " ";
                su += rf::exp(U[k], 6) + " ";
                sv += rf::exp(V[k], 6) + " ";
            }
            st += "\n";
            su += "\n";
            sv += "\n";
        }
        const std::string ext = "0 " + std::to_string(nx - 1) + " 0 " + std::to_string(ny - 1) + " 0 0";
        std::string s = "<?xml version=\"1.0\"?>\n";
        s += "<VTKFile type=\"ImageData\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
        s += "  <ImageData WholeExtent=\"" + ext + "\" Origin=\"0 0 0\" Spacing=\"1 1 1\">\n";
        s += "    <Piece Extent=\"" + ext + "\">\n";
        s += "      <PointData Scalars=\"Temperature\">\n";
        s += "        <DataArray type=\"Float64\" Name=\"Temperature\" format=\"ascii\">\n";
        s += st + "        </DataArray>\n";
        s += "        <DataArray type=\"Float64\" Name=\"Ux\" format=\"ascii\">\n";
        s += su + "        </DataArray>\n";
        s += "        <DataArray type=\"Float64\" Name=\"Uy\" format=\"ascii\">\n";
        s += sv + "        </DataArray>\n";
        s += "      </PointData>\n      <CellData>\n      </CellData>\n    </Piece>\n  </ImageData>\n</VTKFile>\n";
        oks[2] = write_text(join(args.out, "snapshot.vti"), s, errs[2]);
    }
    oks[3] = cav_snapshot_write_fields(join(args.out, "snapshot.bin").c_str(), nx, ny, R.data(), U.data(), V.data(),
                                       T.data()) == CAV_OK;
    if (!oks[3]) errs[3] = cav_last_error(nullptr);
    {  // write_summary_json (:306-360)
        std::string s = "{\n";
        s += "  \"case\": \"differentially_heated_cavity_2d\",\n";
        s += "  \"ra\": " + rf::exp_short(args.ra) + ",\n";
        s += "  \"cs\": " + rf::display(args.cs) + ",\n";
        s += "  \"grid\": [{\"nx\": " + std::to_string(nx) + ", \"ny\": " + std::to_string(ny) + "}],\n";
        s += "  \"aspect_ratio\": " + rf::fixed(double(ny - 1) / double(nx - 1), 4) + ",\n";
        s += "  \"steps\": " + std::to_string(args.steps) + ",\n";
        s += "  \"time_samples\": " + std::to_string(n_samples) + ",\n";
        s += "  \"nusselt_hot\": " + rf::fixed(nuc, 4) + ",\n";
        s += "  \"nusselt_cold\": " + rf::fixed(nuf, 4) + ",\n";
        s += "  \"nusselt_volume\": " + rf::fixed(fin.nusselt_volume, 4) + ",\n";
        s += "  \"wmax_z05\": " + rf::fixed(wmax_mid, 5) + ",\n";
        s += "  \"x_wmax_z05\": " + rf::fixed(x_mid, 5) + ",\n";
        s += "  \"wmax_z075\": " + rf::fixed(wmax_075, 5) + ",\n";
        s += "  \"x_wmax_z075\": " + rf::fixed(x_075, 5) + ",\n";
        s += "  \"y_plus_hot\": " + rf::fixed(yplus, 3) + ",\n";
        s += "  \"references_thesis_tab27\": {\n";
        s += "    \"nuc_snd\": 102.0,\n";
        s += "    \"nuc_les_these\": [100.2, 100.5],\n";
        s += "    \"wmax_z05\": [0.22, 0.24],\n";
        s += "    \"x_wmax_z05\": 0.004,\n";
        s += "    \"wmax_z075\": [0.11, 0.17],\n";
        s += "    \"x_wmax_z075\": 0.005,\n";
        s += "    \"s_half\": [1.10, 1.20]\n";
        s += "  }\n";
        s += "}\n";
        oks[4] = write_text(join(args.out, "summary.json"), s, errs[4]);
    }
    oks[5] = write_text(join(args.out, "progress.log"), log_text(log_lines), errs[5]);
    for (int i = 0; i < 6; ++i)
        if (!oks[i]) {
            err_line("Erreur d'écriture : " + errs[i]);
            return 5;
        }
    if (args.dynamic_smag) {
        double st[4];
        ck(cav_dynamic_sgs_stats(h, st), "cav_dynamic_sgs_stats");
        double nt_sum = 0.0, nt_max = 0.0;
        for (double v : nut_m) {
            nt_sum += v;
            nt_max = std::fmax(nt_max, std::fabs(v));
        }
        std::string s = "{\n";
        s += "  \"dynamic_smag\": true,\n";
        s += "  \"smag_alpha\": " + rf::display(args.smag_alpha) + ",\n";
        s += "  \"eta_test\": " + rf::display(args.eta_test) + ",\n";
        s += "  \"nu_sm_min\": " + rf::display(args.nu_sm_min) + ",\n";
        s += "  \"cs_dyn_mean\": " + rf::fixed(st[0], 6) + ",\n";
        s += "  \"cs_dyn_max\": " + rf::fixed(st[1], 6) + ",\n";
        s += "  \"kappa_dyn_mean\": " + rf::fixed(st[2], 6) + ",\n";
        s += "  \"kappa_dyn_max\": " + rf::fixed(st[3], 6) + ",\n";
        s += "  \"nu_t_mean\": " + rf::exp(nt_sum / double(n), 6) + ",\n";
        s += "  \"nu_t_max\": " + rf::exp(nt_max, 6) + "\n";
        s += "}";
        std::string e;
        if (!write_text(join(args.out, "dynamic_sgs.json"), s, e))
            err_line("Warning : dynamic_sgs.json non écrit : " + e);
        out_line("LES dynamique : cs_dyn_mean = " + rf::fixed(st[0], 4) + " | cs_dyn_max = " + rf::fixed(st[1], 4) +
                 " (clamp [0, 0.04])");
    }
    out_line("--- Résultats (champs moyens) ---");
    const double nu_target = nusselt_trias_2d(args.ra);
    const double ecart = std::fabs((nuc - nu_target) / nu_target) * 100.0;
    out_line("Nuc = " + rf::fixed(nuc, 4) + " | Nuf = " + rf::fixed(nuf, 4) + " | cible Trias 2D (Ra = " +
             rf::exp(args.ra, 2) + ") = " + rf::fixed(nu_target, 2) + " | écart = " + rf::fixed(ecart, 1) + "%");
    out_line("w_max(z=0.5) = " + rf::fixed(wmax_mid, 5) + " en x = " + rf::fixed(x_mid, 5) +
             " (global) ; BL chaude : " + rf::fixed(wmax_mid_hot, 5) + " en x = " + rf::fixed(x_mid_hot, 5) +
             " (cible ≈ 0.23 en x ≈ 0.004)");
    out_line("w_max(z=0.75) = " + rf::fixed(wmax_075, 5) + " en x = " + rf::fixed(x_075, 5) +
             " (global) ; BL chaude : " + rf::fixed(wmax_075_hot, 5) + " en x = " + rf::fixed(x_075_hot, 5) +
             " (cible ≈ 0.11 en x ≈ 0.005)");
    out_line("y+ (paroi chaude) = " + rf::fixed(yplus, 3) + " | S^(1/2) = " + rf::fixed(s_half, 4));
    out_line("Artefacts écrits dans " + args.out);
    cav_destroy(h);
    return 0;
}

// ---- run_octree, src/main.rs:447-720 ------------------------------------------
int run_octree(const Args& args) {
    out_line("=== Cavité DHC 2D octree (Étape B, porte V2) ===");
    out_line("Grossier : " + std::to_string(args.nx0) + "×" + std::to_string(args.ny0) + " | BL fine : " +
             std::to_string(args.bl_width) + " cellules grossières ×2 parois (équiv. uniforme " +
             std::to_string(2 * args.bl_width) + "×" + std::to_string(args.ny0) + ") | Ra = " + rf::exp(args.ra, 3) +
             " | Pr = " + rf::display(args.pr) + " | jobs = " + std::to_string(args.jobs) + " | ξ_odd = " +
             (args.odd_exact ? "exact (τ⁻)" : "1/2 (approx.)"));
    if (args.has_nu)
        out_line("Étape H : nu forcé = " + rf::display(args.nu) + " (bypass calage utarget = " +
                 rf::display(args.utarget) + ")");
    else if (args.utarget != OCT_UTARGET)
        out_line("Étape H : calage ν via utarget = " + rf::display(args.utarget));
    if (args.nu_start_mult > 1.0) {
        const long long spin_up = std::max<long long>(args.ny0 / 10, 2000);
        out_line("Étape H : rampe de viscosité exponentielle nu-start-mult = " + rf::display(args.nu_start_mult) +
                 " (tau_ramp = 1000 pas, terminée ~5000 pas) + rampe beta linéaire sur " + std::to_string(spin_up) +
                 " pas (spin-up)");
        if (args.sample_start < 5000)
            err_line("WARNING : rampe de viscosité terminée ~5000 pas mais sample-start = " +
                     std::to_string(args.sample_start) +
                     " : augmentez --sample-start (> 5000) pour ne pas moyenner pendant la rampe");
    }
    const int prec = octree_precision(args.precision);
    if (prec < 0) {
        err_line("Error: unknown --precision '" + args.precision + "' for the octree solver");
        return 1;
    }
    cav_octree_params p;
    cav_octree_default_params(&p);
    p.nx0 = int32_t(args.nx0);
    p.ny0 = int32_t(args.ny0);
    p.bl_width = int32_t(args.bl_width);
    p.ra = args.ra;
    p.pr = args.pr;
    p.utarget = args.utarget;
    p.seed = args.seed;
    p.jobs = int32_t(args.jobs);
    p.odd_exact = args.odd_exact ? 1 : 0;
    p.levels = int32_t(args.levels);
    p.nu_start_mult = args.nu_start_mult;
    p.has_nu_override = args.has_nu ? 1 : 0;
    p.nu_override = args.nu;
    p.precision = prec;
    p.device = args.device;
    cav_octree* h = nullptr;
    int rc = cav_octree_create(&p, &h);
    if (rc != CAV_OK) die_cav("cav_octree_create", rc, cav_octree_last_error(nullptr));
    auto ck = [&](int r, const char* what) {
        if (r != CAV_OK) die_cav(what, r, cav_octree_last_error(h));
    };
    ck(cav_octree_set_dynamic_sgs(h, args.dynamic_smag ? 1 : 0, args.smag_alpha, args.nu_sm_min, args.eta_test),
       "cav_octree_set_dynamic_sgs");
    if (args.dynamic_smag)
        out_line("LES dynamique (Étape D) : alpha_mixte = " + rf::display(args.smag_alpha) + " | nu_sm_min = " +
                 rf::display(args.nu_sm_min) + " | eta_test = " + rf::display(args.eta_test));
    if (args.has_restart) {
        // OCTSNAP1 header: levels (u32 at 12), step (u64 at 16), grid count (u32 at 24)
        FILE* f = std::fopen(args.restart.c_str(), "rb");
        unsigned char hdr[28];
        const bool ok = f && std::fread(hdr, 1, 28, f) == 28 && std::memcmp(hdr, "OCTSNAP1", 8) == 0;
        if (f) std::fclose(f);
        if (!ok) {
            err_line("Erreur de lecture du snapshot " + args.restart + " : bad magic or file too short");
            return 6;
        }
        uint32_t lv, ng;
        uint64_t st;
        std::memcpy(&lv, hdr + 12, 4);
        std::memcpy(&st, hdr + 16, 8);
        std::memcpy(&ng, hdr + 24, 4);
        out_line("Restart depuis " + args.restart + " : snapshot levels=" + std::to_string(lv) + " (" +
                 std::to_string(ng) + " grilles), pas " + std::to_string(st) +
                 " — injection des champs du solveur octree");
        if (cav_octree_restart_from_snapshot(h, args.restart.c_str()) != CAV_OK) {
            err_line(std::string("Erreur de restart : ") + cav_octree_last_error(h));
            return 6;
        }
    }
    cav_octree_info info;
    ck(cav_octree_get_info(h, &info), "cav_octree_get_info");
    const double beta_f = 0.5 * info.beta_eff_coarse;
    const long long n0 = args.nx0 * args.ny0;
    out_line("Unités réseau : nu = " + rf::fixed(info.nu, 6) + " | alpha = " + rf::fixed(info.alpha, 6) +
             " | tau+ = " + rf::fixed(info.tau_plus[0], 4) + "/" + rf::fixed(info.tau_plus[1], 4) +
             (args.levels == 3 ? "/" + rf::fixed(info.tau_plus[2], 4) : std::string()) +
             " | beta_eff = " + rf::exp(info.beta_eff_coarse, 4) + "/" + rf::exp(beta_f, 4) +
             (args.levels == 3 ? "/" + rf::exp(0.25 * info.beta_eff_coarse, 4) : std::string()) + " | " +
             std::to_string(args.levels) + " niveaux | " + std::to_string(info.n_nodes_total) +
             " nœuds (grossier " + std::to_string(n0) + " + fins " + std::to_string(info.n_nodes_total - n0) + ")");
    const double lz0 = double(args.ny0 - 1);
    out_line("Ra vérifié depuis unités réseau (grossier) : " +
             rf::exp(info.beta_eff_coarse * (lz0 * lz0 * lz0) / (info.nu * info.alpha), 4) + " (cible " +
             rf::exp(args.ra, 4) + ")");
    {
        std::string e;
        if (!create_dir_all(args.out, e)) {
            err_line("Impossible de créer " + args.out + " : " + e);
            return 4;
        }
    }
    std::vector<std::string> log_lines;
    double nuc_sum = 0.0, nuf_sum = 0.0, nucl0_sum = 0.0, nufine_sum = 0.0;
    long long nuc_n = 0;
    double noise_max = 0.0, noise_iface_max = 0.0;
    const auto t0 = std::chrono::steady_clock::now();
    const std::string snap_path = args.snapshot_every > 0 ? join(args.out, "snapshot.bin") : "";
    for (long long s = 0; s < args.steps;) {
        const long long step = next_event(s, args.steps, args.progress_every, args.sample_start, args.sample_every,
                                          args.snapshot_every, true);
        ck(cav_octree_step(h, step - s + 1), "cav_octree_step");
        s = step + 1;
        const bool sample = step >= args.sample_start && (step - args.sample_start) % args.sample_every == 0;
        const bool progress = step % args.progress_every == 0 || step + 1 == args.steps;
        cav_octree_diag_out d{};
        if (sample || progress) ck(cav_octree_diag(h, &d), "cav_octree_diag");
        if (sample) {
            nuc_sum += d.nu_hot;
            nuf_sum += d.nu_cold;
            nucl0_sum += d.nu_hot_link0;
            nufine_sum += d.nu_hot_fine;
            ++nuc_n;
        }
        if (progress) {
            noise_max = std::fmax(noise_max, d.max_rho_dev);
            noise_iface_max = std::fmax(noise_iface_max, d.max_rho_dev_ifaces);
            std::string dyn;
            if (args.dynamic_smag) {
                double st[14];
                ck(cav_octree_dynamic_stats(h, st), "cav_octree_dynamic_stats");
                dyn = " | cs_dyn = " + rf::fixed(st[0], 4) + " | kap_dyn = " + rf::fixed(st[2], 4) +
                      " | nu_t_max = " + rf::exp(st[4], 3);
            }
            const std::string msg = "step " + rf::right(std::to_string(step), 7) + " | max_rho_dev = " +
                                    rf::exp(d.max_rho_dev, 3) + " | max_rho_dev_ifaces = " +
                                    rf::exp(d.max_rho_dev_ifaces, 3) + " | masse = " + rf::fixed(d.mass, 6) +
                                    " | Nuc = " + rf::fixed(d.nu_hot, 4) + " | Nuc_link0 = " +
                                    rf::fixed(d.nu_hot_link0, 4) + " | Nuf = " + rf::fixed(d.nu_cold, 4) +
                                    " | Nu_fin = " + rf::fixed(d.nu_hot_fine, 4) + " | max_u = " +
                                    rf::fixed(d.max_u, 5) + dyn;
            out_line(msg);
            log_lines.push_back(msg);
            // check_guards, src/octree/solver.rs:1019-1038
            std::string abort_msg;
            if (d.max_u > MAX_U_ABORT)
                abort_msg = "AVORT : max_u = " + rf::fixed(d.max_u, 5) + " dépasse le garde-fou " +
                            rf::fixed(MAX_U_ABORT, 2) + " (Ma_local = max_u·√3 ≈ " +
                            rf::fixed(d.max_u * std::sqrt(3.0), 3) + ")";
            else if (d.finite != 1.0)
                abort_msg = "DIVERGENCE détectée (valeurs non finies).";
            if (!abort_msg.empty()) {
                err_line(abort_msg);
                log_lines.push_back(abort_msg);
                std::string e;
                std::string txt;
                for (size_t i = 0; i < log_lines.size(); ++i) txt += (i ? "\n" : "") + log_lines[i];
                write_text(join(args.out, "progress.log"), txt + "\n", e);
                return 2;
            }
        }
        if (args.snapshot_every > 0 && (step + 1) % args.snapshot_every == 0) {
            if (cav_octree_snapshot_write(h, snap_path.c_str(), uint64_t(step)) != CAV_OK) {
                err_line("Erreur d'export du snapshot au pas " + std::to_string(step) + " : " +
                         cav_octree_last_error(h));
                return 5;
            }
            out_line("snapshot exporté au pas " + std::to_string(step));
        }
    }
    if (args.snapshot_every > 0) {
        if (cav_octree_snapshot_write(h, snap_path.c_str(), uint64_t(args.steps)) != CAV_OK) {
            err_line(std::string("Erreur d'export du snapshot final : ") + cav_octree_last_error(h));
            return 5;
        }
        out_line("snapshot final exporté au pas " + std::to_string(args.steps - 1));
    }
    ck(cav_octree_sync(h), "cav_octree_sync");
    const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    out_line("Simulation terminée en " + rf::fixed(elapsed, 1) + " s (" +
             rf::fixed(double(args.steps) / elapsed / 1000.0, 1) + "k pas/s)");
    if (nuc_n == 0) {
        err_line("Aucun échantillon moyenné : sample_start ≥ steps ?");
        return 3;
    }
    const double nuc_mean = nuc_sum / double(nuc_n), nuf_mean = nuf_sum / double(nuc_n);
    const double nucl0_mean = nucl0_sum / double(nuc_n), nufine_mean = nufine_sum / double(nuc_n);
    const double nuc_ref = 2.3585, nucl0_ref = 1.3660;
    const double ecart = std::fabs((nuc_mean - nuc_ref) / nuc_ref) * 100.0;
    const std::string summary =
        "--- Bilan (moyenné sur " + std::to_string(nuc_n) + " échantillons, fenêtre " +
        std::to_string(args.sample_start) + "→" + std::to_string(args.steps) + ") ---\n" +
        "Nuc (2ᵉ liaison) = " + rf::fixed(nuc_mean, 4) + " | écart like-for-like vs " + rf::display(nuc_ref) + " = " +
        rf::fixed(ecart, 1) + " %\n" + "Nuc_link0 (1ʳᵉ liaison) = " + rf::fixed(nucl0_mean, 4) +
        " | Nuf = " + rf::fixed(nuf_mean, 4) + " | Nu_fin (bloc chaud) = " + rf::fixed(nufine_mean, 4) + "\n" +
        "Références uniforme Ra=1e6 : 2ᵉ liaison = " + rf::display(nuc_ref) + " | 1ʳᵉ liaison = " +
        rf::display(nucl0_ref) + "\n" + "Bruit acoustique (max sur la run) : max|ρ−ρ̄| = " + rf::exp(noise_max, 3) +
        " | interfaces = " + rf::exp(noise_iface_max, 3) + "\n" +
        "PORTE V2 (écart Nuc ≤ 5 %) : " + (ecart <= 5.0 ? "PASS" : "FAIL");
    out_line(summary);
    log_lines.push_back(summary);
    std::string txt;
    for (size_t i = 0; i < log_lines.size(); ++i) txt += (i ? "\n" : "") + log_lines[i];
    std::string e;
    write_text(join(args.out, "progress.log"), txt + "\n", e);
    out_line("Artefacts écrits dans " + args.out);
    cav_octree_destroy(h);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    bool help = false;
    Args args;
    try {
        args = parse_args(argc, argv, help);
    } catch (const ArgError& e) {
        std::fprintf(stderr, "Error: %s\n\n%s", e.msg.c_str(), USAGE);
        return 1;
    }
    if (help) {
        std::fputs(USAGE, stderr);
        return 0;
    }
    return args.mode == Mode::Uniform ? run_uniform(args) : run_octree(args);
}
