// mem_cuda.cpp — drop-in replacement of cudaturbo's mem_cuda CLI on the dns2d C ABI.
//
// Same command line, environment, signals, stdout lines and output files as the reference
// driver (cuda/mem_cuda.cu:1664-2082):
//   mem_cuda [N Re K0 STEPS CFL UPDATE ADAPT_VISC [restart.bin|MOV] [MOV]]
//   mem_cuda RESTART <output folder>            (reads meta.csv + restart.bin of the folder)
//   env: PHASE_TIMING, BENCH_WARMUP_STEPS, RESTART_STEPS, NVIDIA_SMI, MOV, MOV_DIR
//   new env (no counterpart): IC=k4 with SEED=<n> starts from the seeded
//   k^4 exp(-2 (k/K0)^2) spectrum instead of PAO-k^-3.
// Signals (polled once per step, cuda/mem_cuda.cu:44-135): SIGUSR1 save and continue,
// SIGRTMIN save + restart.bin and continue, SIGUSR2 pause / SIGCONT resume, SIGHUP and SIGTERM
// save and exit, SIGINT exit without saving; exit code 128 + signal.
#include "dns2d.h"
#include "png_writer.h"

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cctype>
#include <cmath>
#include <csignal>
#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <thread>
#include <vector>

#include <dirent.h>
#include <sys/stat.h>

namespace {

volatile std::sig_atomic_t g_exit_requested = 0, g_exit_signal = 0, g_save_requested = 0,
                           g_save_restart_requested = 0, g_pause_requested = 0, g_resume_requested = 0;

void on_exit_signal(int sig)
{
    g_exit_requested = 1;
    g_exit_signal = sig;
}
void on_save(int) { g_save_requested = 1; }
void on_save_restart(int) { g_save_restart_requested = 1; }
void on_pause(int) { g_pause_requested = 1; }
void on_resume(int) { g_resume_requested = 1; }

void install_signals()
{
    std::signal(SIGHUP, on_exit_signal);
    std::signal(SIGUSR1, on_save);
    std::signal(SIGUSR2, on_pause);
    std::signal(SIGCONT, on_resume);
    std::signal(SIGRTMIN, on_save_restart);
    std::signal(SIGINT, on_exit_signal);
    std::signal(SIGTERM, on_exit_signal);
}

void ignore_signals()
{
    for (int s : {SIGHUP, SIGUSR1, SIGUSR2, SIGCONT, SIGINT, SIGTERM}) std::signal(s, SIG_IGN);
    std::signal(SIGRTMIN, SIG_IGN);
}

const char *signal_name(int sig)
{
    if (sig == SIGRTMIN) return "SIGRTMIN";
    switch (sig) {
    case SIGHUP: return "SIGHUP";
    case SIGUSR1: return "SIGUSR1";
    case SIGUSR2: return "SIGUSR2";
    case SIGCONT: return "SIGCONT";
    case SIGINT: return "SIGINT";
    case SIGTERM: return "SIGTERM";
    default: return "signal";
    }
}

bool flag_on(const char *raw)
{
    if (!raw || !raw[0]) return false;
    std::string s(raw);
    for (auto &c : s) c = (char)std::tolower((unsigned char)c);
    if (s == "true" || s == "yes" || s == "on") return true;
    return std::atoi(raw) != 0;
}

bool iequals(const char *a, const char *b)
{
    if (!a || !b) return false;
    for (; *a && *b; ++a, ++b)
        if (std::toupper((unsigned char)*a) != std::toupper((unsigned char)*b)) return false;
    return !*a && !*b;
}

std::string sci_no_plus(float x)
{
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.0E", (double)x);
    std::string s(buf);
    const size_t p = s.find("E+");
    if (p != std::string::npos) s.replace(p, 2, "E");
    return s;
}

bool make_dir(const std::string &path)
{
    if (mkdir(path.c_str(), 0775) == 0 || errno == EEXIST) return true;
    std::fprintf(stderr, "Failed to create output folder %s: %s\n", path.c_str(), std::strerror(errno));
    return false;
}

std::string join(const std::string &a, const char *b) { return a + "/" + b; }

// ---------------------------------------------------------------------------------------
// movie frames (cuda/mem_cuda.cu:245-330, :1834-1846, :1899-1910; cuda/color_cuda.cu:269-375)
// ---------------------------------------------------------------------------------------

// "MOV" among the optional arguments enables frames unless the MOV variable says otherwise;
// without the argument the MOV variable alone decides (cuda/mem_cuda.cu:245-255)
bool mov_flag(int argc, char **argv, int first)
{
    const char *raw = std::getenv("MOV");
    for (int i = first; i < argc; ++i)
        if (iequals(argv[i], "MOV")) raw = (raw && raw[0]) ? raw : "1";
    return flag_on(raw);
}

bool make_dirs(const std::string &path)
{
    for (size_t p = 1; p <= path.size(); ++p) {
        if (p < path.size() && path[p] != '/') continue;
        const std::string part = path.substr(0, p);
        if (mkdir(part.c_str(), 0775) != 0 && errno != EEXIST) {
            std::fprintf(stderr, "Failed to create movie folder %s: %s\n", part.c_str(), std::strerror(errno));
            return false;
        }
    }
    return true;
}

// <MOV_DIR or ./movies>/cuda_<N>_<K0>_<Re>_<CFL %.3f>_U<UPDATE>
std::string movie_folder_name(int N, float K0, float Re, float CFL, int update)
{
    const char *root = std::getenv("MOV_DIR");
    char cfl[64];
    std::snprintf(cfl, sizeof(cfl), "%.3f", (double)CFL);
    return std::string(root && root[0] ? root : "movies") + "/cuda_" + std::to_string(N) + "_" +
           std::to_string((int)K0) + "_" + sci_no_plus(Re) + "_" + cfl + "_U" + std::to_string(update);
}

// highest k among the folder's omega_inferno_<digits>.png files, 0 when there are none: a continued
// run appends frames after the ones already there
int last_movie_frame(const std::string &folder)
{
    DIR *d = opendir(folder.c_str());
    if (!d) return 0;
    static const char pre[] = "omega_inferno_", suf[] = ".png";
    const size_t lp = sizeof(pre) - 1, ls = sizeof(suf) - 1;
    int last = 0;
    while (const dirent *e = readdir(d)) {
        const std::string n(e->d_name);
        if (n.size() <= lp + ls || n.compare(0, lp, pre) != 0 || n.compare(n.size() - ls, ls, suf) != 0) continue;
        const std::string digits = n.substr(lp, n.size() - lp - ls);
        if (!std::all_of(digits.begin(), digits.end(), [](char c) { return std::isdigit((unsigned char)c) != 0; }))
            continue;
        last = std::max(last, std::atoi(digits.c_str()));
    }
    closedir(d);
    return last;
}


// one frame of the vorticity plane (comp 2 of the physical planes, filled by dns2d_om2phys)
bool save_movie_frame(dns2d_state *s, const PngWriter &png, const std::string &path, int F)
{
    int w = 0, h = 0;
    double sigma = 0.0;
    dns2d_movie_frame(s, 2, F, nullptr, &w, &h, nullptr);
    std::vector<unsigned char> rgb((size_t)w * h * 3);
    const int rc = dns2d_movie_frame(s, 2, F, rgb.data(), &w, &h, &sigma);
    if (rc) {
        std::fprintf(stderr, "dns2d_movie_frame failed: %s (%s)\n", dns2d_strerror(rc), dns2d_last_error(s));
        return false;
    }
    if (!png.write(path, w, h, rgb.data())) return false;
    std::printf("[MOV] Wrote %s (Inferno PNG, %dx%d, F=%d, comp=%d, sigma=%d)\n", path.c_str(), w, h, F, 2, (int)sigma);
    return true;
}

void die(dns2d_state *s, int rc, const char *what)
{
    std::fprintf(stderr, "%s failed: %s (%s)\n", what, dns2d_strerror(rc), s ? dns2d_last_error(s) : "");
}

// ---------------------------------------------------------------------------------------
// metrics / meta CSV (cuda/mem_cuda.cu:482-567, :954-994)
// ---------------------------------------------------------------------------------------
struct MetricsRow {
    int N, K0;
    double Re, CFL, VISC, DT;
    int STEPS, PALIN, SIG;
    double TIME, MINUTES, FPS;
};

struct AdaptVisc {
    double e_int = 0.0, e_prev = 0.0, target = 20.0, palin_filt = 0.0, palin_filt_1 = 0.0;
};

double re_from_nk0(int N, double K0)
{
    return std::pow(10.0, 1.066240 * std::log10((double)N) - 0.083911 * std::log10(K0) + 1.286396);
}

// PD controller on the filtered palinstrophy ratio (cuda/mem_cuda.cu:458-528)
void adapt_visc(dns2d_scalars &sc, AdaptVisc &A, double pal)
{
    const double p_raw = 10000.0 * pal;
    const double alpha = 1.0 / (5.0 + 1.0);
    if (A.palin_filt == 0.0) {
        A.palin_filt_1 = p_raw;
        A.palin_filt = p_raw;
    } else {
        A.palin_filt_1 += alpha * (p_raw - A.palin_filt_1);
        A.palin_filt += alpha * (A.palin_filt_1 - A.palin_filt);
    }
    const double e = (A.palin_filt - A.target) / A.target;
    if (std::fabs(e) < 0.001) return;
    const double de = e - A.e_prev;
    A.e_prev = e;
    double u = 0.25 * e + 25.0 * de;
    u = std::max(-0.01, std::min(0.01, u));
    const double nu_new = (double)sc.visc * std::exp(u);
    const double Re0 = re_from_nk0(sc.N, (double)sc.K0);
    const double Re_eff = std::max(Re0 / 1000.0, std::min(1000.0 * Re0, 1.0 / nu_new));
    sc.Re = (float)Re_eff;
    sc.visc = (float)(1.0 / Re_eff);
}

MetricsRow make_row(const dns2d_scalars &sc, double pal, double sigma, double elapsed, int start_iter)
{
    const int steps = sc.it - start_iter;
    return MetricsRow{sc.N, (int)sc.K0, (double)sc.Re, (double)sc.cflnum, (double)sc.visc, (double)sc.dt, sc.it,
                      (int)(10000.0 * pal), (int)sigma, (double)sc.t, elapsed / 60.0,
                      elapsed > 0.0 ? (double)steps / elapsed : 0.0};
}

void append_row(std::vector<MetricsRow> &rows, const MetricsRow &r)
{
    if (!rows.empty() && rows.back().STEPS == r.STEPS) rows.back() = r;
    else rows.push_back(r);
}

bool save_metrics(const std::vector<MetricsRow> &rows, const std::string &path)
{
    FILE *fp = std::fopen(path.c_str(), "w");
    if (!fp) {
        std::perror("saveMetricsCsv: fopen");
        return false;
    }
    std::fprintf(fp, "N,K0,Re,CFL,VISC,DT,STEPS,PALIN,SIG,TIME,MINUTES,FPS\n");
    for (const MetricsRow &r : rows)
        std::fprintf(fp, "%d,%d,%.17g,%.17g,%.17g,%.17g,%d,%d,%d,%.17g,%.17g,%.17g\n", r.N, r.K0, r.Re, r.CFL,
                     r.VISC, r.DT, r.STEPS, r.PALIN, r.SIG, r.TIME, r.MINUTES, r.FPS);
    std::fclose(fp);
    std::printf("[CSV] Wrote %s (metrics, %zu rows)\n", path.c_str(), rows.size());
    return true;
}

bool save_meta(const dns2d_scalars &sc, const std::string &path, int update, double sigma, double pal,
               double minutes, double fps)
{
    FILE *fp = std::fopen(path.c_str(), "w");
    if (!fp) {
        std::perror("saveMetaCsv: fopen");
        return false;
    }
    char ts[32];
    std::time_t now = std::time(nullptr);
    std::tm tm_now{};
    localtime_r(&now, &tm_now);
    std::strftime(ts, sizeof(ts), "%Y-%m-%d %H:%M", &tm_now);
    std::fprintf(fp, "timestamp,N,K0,Re,CFL,visc,T,IT,Update,sigma,10K_pal_over_Zkmax2,minutes,FPS,backend\n");
    std::fprintf(fp, "%s,%d,%.9g,%.9g,%.9g,%.9g,%.9g,%d,%d,%d,%.9g,%.9g,%.9g,CUDA\n", ts, sc.N, (double)sc.K0,
                 (double)sc.Re, (double)sc.cflnum, (double)sc.visc, (double)sc.t, sc.it, update, (int)sigma,
                 10000.0 * pal, minutes, fps);
    std::fclose(fp);
    std::printf("[CSV] Wrote %s (metadata)\n", path.c_str());
    return true;
}

// ---------------------------------------------------------------------------------------
// PGM dumps (cuda/dns_cuda.cu:643-807): min/max of finite values, optional percentile clip
// through an 8192-bin histogram, pixels round(1 + 254 (v - lo) / (hi - lo)) clamped to 1..255
// ---------------------------------------------------------------------------------------
void field_range(const std::vector<float> &h, bool clipped, double lo_pct, double hi_pct, float &minv, float &maxv,
                 float &lo, float &hi)
{
    minv = 1.0e30f;
    maxv = -1.0e30f;
    size_t finite = 0;
    for (float v : h) {
        if (!std::isfinite(v)) continue;
        minv = std::min(minv, v);
        maxv = std::max(maxv, v);
        ++finite;
    }
    if (finite == 0) minv = maxv = 0.0f;
    lo = minv;
    hi = maxv;
    if (!clipped || finite == 0 || maxv - minv <= 1.0e-12f) return;
    lo_pct = std::max(0.0, std::min(1.0, lo_pct));
    hi_pct = std::max(0.0, std::min(1.0, hi_pct));
    if (!(lo_pct < hi_pct)) return;
    const int bins = 8192;
    std::vector<size_t> hist(bins, 0);
    const double inv = (double)(bins - 1) / (double)(maxv - minv);
    for (float v : h) {
        if (!std::isfinite(v)) continue;
        int b = (int)(((double)v - (double)minv) * inv);
        b = std::max(0, std::min(bins - 1, b));
        ++hist[(size_t)b];
    }
    const size_t lo_rank = (size_t)std::floor(lo_pct * (double)(finite - 1));
    const size_t hi_rank = (size_t)std::floor(hi_pct * (double)(finite - 1));
    int lo_bin = 0, hi_bin = bins - 1;
    size_t acc = 0;
    for (int b = 0; b < bins; ++b) {
        acc += hist[(size_t)b];
        if (acc > lo_rank) {
            lo_bin = b;
            break;
        }
    }
    acc = 0;
    for (int b = 0; b < bins; ++b) {
        acc += hist[(size_t)b];
        if (acc > hi_rank) {
            hi_bin = b;
            break;
        }
    }
    const double w = (double)(maxv - minv) / (double)bins;
    lo = (float)((double)minv + w * (double)lo_bin);
    hi = (float)((double)minv + w * (double)(hi_bin + 1));
    if (!(hi > lo)) {
        lo = minv;
        hi = maxv;
    }
}

bool dump_pgm(dns2d_state *s, int comp, const std::string &path, bool clipped, int L)
{
    std::vector<float> h((size_t)L * L);
    int rc = dns2d_get_phys(s, comp, h.data());
    if (rc) {
        die(s, rc, "dns2d_get_phys");
        return false;
    }
    float minv, maxv, lo, hi;
    field_range(h, clipped, 0.001, 0.999, minv, maxv, lo, hi);
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) {
        std::perror("fopen");
        return false;
    }
    std::fprintf(f, "P5\n%d %d\n255\n", L, L);
    const float range = hi - lo;
    std::vector<unsigned char> px(h.size());
    for (size_t i = 0; i < h.size(); ++i) {
        if (range <= 1e-12f) {
            px[i] = 128;
            continue;
        }
        const float v = h[i];
        const float norm = std::isfinite(v) ? (v - lo) / range : 0.5f;
        int p = (int)(1.0f + norm * 254.0f + 0.5f);
        px[i] = (unsigned char)std::max(1, std::min(255, p));
    }
    std::fwrite(px.data(), 1, px.size(), f);
    std::fclose(f);
    if (clipped)
        std::printf("[DUMP] Wrote %s (PGM, %dx%d, comp=%d, min=%g, max=%g, clip=%g..%g)\n", path.c_str(), L, L, comp,
                    (double)minv, (double)maxv, (double)lo, (double)hi);
    else
        std::printf("[DUMP] Wrote %s (PGM, %dx%d, comp=%d, min=%g, max=%g)\n", path.c_str(), L, L, comp, (double)minv,
                    (double)maxv);
    return true;
}

// energy_spectrum.csv (cuda/mem_cuda.cu:575-649)
bool save_spectrum(dns2d_state *s, const std::string &path, int L)
{
    const int nbins = std::max(32, 2 * L);
    std::vector<double> e((size_t)nbins);
    std::vector<int> c((size_t)nbins);
    int rc = dns2d_velocity_spectrum_bins(s, e.data(), c.data(), nbins);
    if (rc) {
        die(s, rc, "spectrum");
        return false;
    }
    FILE *fp = std::fopen(path.c_str(), "w");
    if (!fp) {
        std::perror("saveEnergySpectrumUvCsv: fopen");
        return false;
    }
    const double r_max = std::sqrt(2.0);
    std::fprintf(fp, "normalized_radius,shell_sum_energy,count\n");
    for (int i = 0; i < nbins; ++i)
        if (c[(size_t)i] > 0 && e[(size_t)i] > 0.0) {
            const double r0 = r_max * i / nbins, r1 = r_max * (i + 1) / nbins;
            std::fprintf(fp, "%.17g,%.17g,%d\n", 0.5 * (r0 + r1), e[(size_t)i], c[(size_t)i]);
        }
    std::fclose(fp);
    std::printf("[CSV] Wrote %s (energy spectrum, %d bins)\n", path.c_str(), nbins);
    return true;
}

std::string folder_name(const dns2d_scalars &sc, int N, float K0, float Re, float CFL)
{
    char cfl[64];
    std::snprintf(cfl, sizeof(cfl), "%.2f", (double)CFL);
    return "output_" + std::to_string(N) + "_" + std::to_string((int)K0) + "_" + sci_no_plus(Re) + "_" + cfl + "_" +
           std::to_string(sc.it);
}

// dump sequence of cuda/mem_cuda.cu:1396-1449
bool dump_outputs(dns2d_state *s, const std::vector<MetricsRow> &rows, const std::string &folder, int update,
                  double elapsed, double fps)
{
    if (!make_dir(folder)) return false;
    std::printf("[SAVE] Dumping fields to folder: %s\n", folder.c_str());
    dns2d_scalars sc;
    dns2d_get_scalars(s, &sc);
    const int L = sc.NX_full;
    if (dns2d_velocity_phys(s)) return false;
    dump_pgm(s, 0, join(folder, "u_velocity.pgm"), false, L);
    dump_pgm(s, 1, join(folder, "v_velocity.pgm"), false, L);
    dns2d_kinetic(s);
    dump_pgm(s, 2, join(folder, "kinetic.pgm"), false, L);
    dns2d_om2phys(s);
    dump_pgm(s, 2, join(folder, "omega.pgm"), true, L);
    double sigma = 0.0, pal = 0.0;
    if (rows.empty()) {
        dns2d_display_sigma(s, 2, &sigma);
        dns2d_palin(s, &pal);
    } else {
        sigma = rows.back().SIG;
        pal = rows.back().PALIN / 10000.0;
    }
    dns2d_stream_func(s);
    dump_pgm(s, 2, join(folder, "stream.pgm"), false, L);
    save_spectrum(s, join(folder, "energy_spectrum.csv"), L);
    save_metrics(rows, join(folder, "metrics.csv"));
    save_meta(sc, join(folder, "meta.csv"), update, sigma, pal, elapsed / 60.0, fps);
    return true;
}

bool read_line(FILE *fp, std::string &line)
{
    char buf[4096];
    if (!std::fgets(buf, sizeof(buf), fp)) return false;
    line = buf;
    while (!line.empty() && (line.back() == '\n' || line.back() == '\r')) line.pop_back();
    return true;
}

// RESTART <folder>: N, K0, Re, CFL and Update from meta.csv (cuda/mem_cuda.cu:374-424)
bool restart_folder_args(const char *folder, int &N, float &Re, float &K0, float &CFL, int &UPDATE, std::string &path)
{
    const std::string meta = std::string(folder) + "/meta.csv";
    FILE *fp = std::fopen(meta.c_str(), "r");
    if (!fp) {
        std::perror("loadRestartFolderArgs: fopen meta.csv");
        return false;
    }
    std::string header, row;
    const bool ok = read_line(fp, header) && read_line(fp, row);
    std::fclose(fp);
    if (!ok) {
        std::fprintf(stderr, "loadRestartFolderArgs: invalid %s\n", meta.c_str());
        return false;
    }
    std::vector<std::string> cols;
    size_t b = 0;
    for (;;) {
        const size_t c = row.find(',', b);
        cols.push_back(row.substr(b, c == std::string::npos ? std::string::npos : c - b));
        if (c == std::string::npos) break;
        b = c + 1;
    }
    if (cols.size() < 9) {
        std::fprintf(stderr, "loadRestartFolderArgs: expected at least 9 columns in %s\n", meta.c_str());
        return false;
    }
    N = std::atoi(cols[1].c_str());
    K0 = (float)std::atof(cols[2].c_str());
    Re = (float)std::atof(cols[3].c_str());
    CFL = (float)std::atof(cols[4].c_str());
    UPDATE = std::atoi(cols[8].c_str());
    if (N <= 0 || K0 <= 0 || Re <= 0 || CFL <= 0 || UPDATE <= 0) {
        std::fprintf(stderr, "loadRestartFolderArgs: invalid run parameters in %s\n", meta.c_str());
        return false;
    }
    path = std::string(folder) + "/restart.bin";
    FILE *r = std::fopen(path.c_str(), "rb");
    if (!r) {
        std::perror("loadRestartFolderArgs: fopen restart.bin");
        return false;
    }
    std::fclose(r);
    return true;
}

void gpu_snapshot(const char *phase)
{
    const char *env = std::getenv("NVIDIA_SMI");
    std::string cmd = (env && env[0]) ? std::string("'") + env + "'" : "nvidia-smi";
    cmd += " --query-gpu=name,persistence_mode,pstate,clocks.sm,clocks.mem,temperature.gpu,power.draw,power.limit "
           "--format=csv,noheader,nounits 2>/dev/null";
    FILE *p = popen(cmd.c_str(), "r");
    std::vector<std::string> lines;
    if (p) {
        char buf[1024];
        while (std::fgets(buf, sizeof(buf), p)) {
            std::string l(buf);
            while (!l.empty() && (l.back() == '\n' || l.back() == '\r')) l.pop_back();
            if (!l.empty()) lines.push_back(l);
        }
        if (pclose(p) != 0) lines.clear();
    }
    if (lines.empty()) {
        std::printf("[GPU] %s: nvidia-smi unavailable\n", phase);
        return;
    }
    std::printf("[GPU] %s fields: name, persistence, pstate, sm_clock_mhz, mem_clock_mhz, temp_c, power_w, "
                "power_limit_w\n",
                phase);
    for (const auto &l : lines) std::printf("[GPU] %s: %s\n", phase, l.c_str());
}

const char *kStatFmt[19] = {" Reynolds n. =%12.1f\n", " Energy      =%12.7f\n", " WiWi        =%12.5f\n",
                            " Epsilon     =%12.7f\n", " a11         =%12.7f\n", " e11         =%12.7f\n",
                            " Time scale  =%12.4f\n", " Kolmogorov  =%12.7f\n", " Viscosity   =%12.7f\n",
                            " dx/Kol.     =%12.7f\n", " 2Pi/Nlamda  =%12.7f\n", " 2Pi/Lux     =%12.7f\n",
                            " 2Pi/Luz     =%12.7f\n", " 2Pi/Lwx     =%12.7f\n", " 2Pi/Lwz     =%12.7f\n",
                            " Deps.       =%12.7f\n", " Ceps2       =%12.7f\n", " E1          =%12.7f\n",
                            " E3          =%12.7f\n"};

}  // namespace

// DUMP <restart.bin> <folder> [UPDATE]: write the files of a signal save (the PGMs,
// energy_spectrum.csv, metrics.csv, meta.csv of cuda/mem_cuda.cu:1396-1449) for the state held in
// a restart file, without stepping.  An addition of this CLI: the reference writes them only from
// a running simulation; this renders any saved state, e.g. the restart.bin of a SIGRTMIN save.
int dump_restart(const char *path, const char *folder, int update)
{
    unsigned char hdr[144];
    FILE *fp = std::fopen(path, "rb");
    if (!fp || std::fread(hdr, 1, sizeof(hdr), fp) < 136) {
        if (fp) std::fclose(fp);
        std::fprintf(stderr, "DUMP: cannot read the header of %s\n", path);
        return 1;
    }
    std::fclose(fp);
    int32_t N = 0;
    float Re = 0.0f, K0 = 0.0f, cfl = 0.0f;
    std::memcpy(&N, hdr + 32, 4);  // Nbase (restart header, cuda/mem_cuda.cu:1019-1054)
    std::memcpy(&Re, hdr + 72, 4);
    std::memcpy(&K0, hdr + 76, 4);
    std::memcpy(&cfl, hdr + 100, 4);
    dns2d_state *s = nullptr;
    int rc = dns2d_create(&s, N, Re, K0, cfl, 0);
    if (rc) {
        std::fprintf(stderr, "DUMP: dns2d_create(N=%d): %s\n", N, dns2d_strerror(rc));
        return 1;
    }
    rc = dns2d_load_restart(s, path);
    if (rc) {
        std::fprintf(stderr, "DUMP: %s: %s\n", dns2d_strerror(rc), dns2d_last_error(s));
        dns2d_destroy(s);
        return 1;
    }
    dns2d_scalars sc;
    dns2d_get_scalars(s, &sc);
    std::printf(" DUMP of %s: N=%d it=%d T=%12.10f\n", path, N, sc.it, (double)sc.t);
    const bool ok = dump_outputs(s, {}, folder, update, 0.0, 0.0);
    dns2d_destroy(s);
    return ok ? 0 : 1;
}

int main(int argc, char **argv)
{
    if (argc > 1 && std::strcmp(argv[1], "DUMP") == 0) {
        if (argc < 4) {
            std::fprintf(stderr, "Usage: %s DUMP restart.bin output_folder [UPDATE]\n", argv[0]);
            return 2;
        }
        return dump_restart(argv[2], argv[3], argc > 4 ? std::atoi(argv[4]) : 0);
    }
    install_signals();
    int N = 512, STEPS = 1001, UPDATE = 100;
    float Re = 10000.0f, K0 = 10.0f, CFL = 0.25f;
    bool ADAPT = false, MOV = false;
    const char *RESTART_PATH = nullptr;
    std::string restart_storage;
    if (argc > 1 && std::strcmp(argv[1], "RESTART") == 0) {
        if (argc < 3) {
            std::fprintf(stderr, "Usage: %s RESTART output_folder\n", argv[0]);
            return 2;
        }
        if (!restart_folder_args(argv[2], N, Re, K0, CFL, UPDATE, restart_storage)) return 1;
        STEPS = 1000000;
        const char *e = std::getenv("RESTART_STEPS");
        if (e && e[0]) STEPS = std::atoi(e);
        RESTART_PATH = restart_storage.c_str();
        MOV = mov_flag(argc, argv, 3);
    } else {
        if (argc > 1) N = std::atoi(argv[1]);
        if (argc > 2) Re = (float)std::atof(argv[2]);
        if (argc > 3) K0 = (float)std::atof(argv[3]);
        if (argc > 4) STEPS = std::atoi(argv[4]);
        if (argc > 5) CFL = (float)std::atof(argv[5]);
        if (argc > 6) UPDATE = std::atoi(argv[6]);
        if (argc > 7) ADAPT = std::atoi(argv[7]) != 0;
        int mov_begin = 8;
        if (argc > 8 && !iequals(argv[8], "MOV")) {
            RESTART_PATH = argv[8];
            mov_begin = 9;
        }
        MOV = mov_flag(argc, argv, mov_begin);
    }
    if (UPDATE <= 0) UPDATE = 100;
    if (STEPS <= 0) STEPS = 1000000;
    const bool phase_timing = flag_on(std::getenv("PHASE_TIMING"));

    std::printf("--- INITIALIZING FPS_CUDA ---\n");
    std::printf(" N=%d, Re=%d, K0=%d, STEPS=%d, CFL=%.3f, UPDATE=%d, ADAPT_VISC=%d, MOV=%d\n", N, (int)Re, (int)K0, STEPS,
                (double)CFL, UPDATE, ADAPT ? 1 : 0, MOV ? 1 : 0);
    if (phase_timing) std::printf("[PHASE] PHASE_TIMING enabled; profiling will synchronize measured phases.\n");
    if (RESTART_PATH) std::printf(" restart=%s\n", RESTART_PATH);
    gpu_snapshot("start");

    dns2d_state *s = nullptr;
    int rc = dns2d_create(&s, N, Re, K0, CFL, 0);
    if (rc) {
        std::printf("dnsCudaCreate failed: %s\n", dns2d_strerror(rc));
        return 1;
    }
    std::printf(" dns2d state: GPU memory ~ %.2f MiB (fused sm_100a kernels, no FFT library work area)\n",
                dns2d_device_bytes(N) / (1024.0 * 1024.0));
    if (phase_timing) dns2d_phase_timing(s, 1);

    const char *ic = std::getenv("IC");
    if (ic && iequals(ic, "k4")) {
        const char *sd = std::getenv("SEED");
        rc = dns2d_init_k4(s, sd ? std::strtoull(sd, nullptr, 10) : 0ULL);
        if (!rc) std::printf(" k4 spectrum initialization OK (seed %s). VISC=%12.7f\n", sd ? sd : "0", 1.0 / Re);
    } else {
        double st[19];
        int seed = 0;
        rc = dns2d_init_pao(s, st, &seed);
        if (!rc) {
            for (int i = 0; i < 19; ++i) std::printf(kStatFmt[i], st[i]);
            std::printf(" PAO seed    =%12d\n", seed);
            dns2d_scalars sc;
            dns2d_get_scalars(s, &sc);
            std::printf(" PAO-kminus3 initialization OK. VISC=%12.7f\n", (double)sc.visc);
        }
    }
    if (rc) {
        die(s, rc, "dnsCudaInit");
        std::printf("dnsCudaInit failed\n");
        dns2d_destroy(s);
        return 1;
    }
    dns2d_scalars sc;
    dns2d_get_scalars(s, &sc);
    sc.cflnum = CFL;
    sc.ifn = 1;
    sc.it = 0;
    sc.dt = 0.0f;
    sc.cn = 1.0f;
    sc.cnm1 = 0.0f;
    dns2d_set_scalars(s, &sc);
    if (RESTART_PATH) {
        rc = dns2d_load_restart(s, RESTART_PATH);
        if (rc) {
            std::fprintf(stderr, "loadRestartBin: %s\n", dns2d_last_error(s));
            dns2d_destroy(s);
            return 1;
        }
        dns2d_get_scalars(s, &sc);
        std::printf("[LOAD] Loaded restart binary %s at iteration %d\n", RESTART_PATH, sc.it);
        N = sc.N;
        K0 = sc.K0;
        CFL = sc.cflnum;
    } else {
        float cflm = 0.0f;
        dns2d_next_dt(s, &cflm);
        dns2d_get_scalars(s, &sc);
        std::printf(" [NEXTDT INIT] CFLM=%12.7f  DT=%12.7f  CN=%12.7f\n", (double)cflm, (double)sc.dt, (double)sc.cn);
        std::printf(" Initial DT=%12.7f  CN=%12.7f\n", (double)sc.dt, (double)sc.cn);
    }

    using clk = std::chrono::steady_clock;
    dns2d_sync(s, 0);
    const auto tbegin = clk::now();
    int warm = UPDATE;
    const char *ew = std::getenv("BENCH_WARMUP_STEPS");
    if (ew && ew[0]) warm = std::max(0, std::atoi(ew));
    dns2d_get_scalars(s, &sc);
    const int start_iter = sc.it;
    AdaptVisc av;
    std::vector<MetricsRow> rows;
    bool interrupted = false, steady_started = false;
    double paused = 0.0, steady_paused0 = 0.0;
    int steady_iter0 = sc.it;
    clk::time_point steady_begin{};
    std::printf("[BENCH] Wall-clock FPS timer starts after initial cudaDeviceSynchronize().\n");
    if (warm > 0) {
        std::printf("[BENCH] Steady FPS will exclude the first %d completed steps (override with BENCH_WARMUP_STEPS).\n",
                    warm);
    } else {
        steady_started = true;
        steady_begin = tbegin;
        std::printf("[BENCH] Steady FPS timer starts immediately (BENCH_WARMUP_STEPS=0).\n");
    }
    auto elapsed_active = [&]() { return std::chrono::duration<double>(clk::now() - tbegin).count() - paused; };
    const int movie_F = dns2d_movie_scale(N);
    std::string movie_folder;
    int movie_frame = 0;
    const PngWriter png;
    if (MOV) {
        movie_folder = movie_folder_name(N, K0, Re, CFL, UPDATE);
        if (!make_dirs(movie_folder)) {
            dns2d_destroy(s);
            return 1;
        }
        movie_frame = last_movie_frame(movie_folder);
        std::printf("[MOV] Saving omega_inferno_%%05d.png every %d steps to %s (F=%d, next=%05d)\n", UPDATE,
                    movie_folder.c_str(), movie_F, movie_frame + 1);
    }
    auto is_diag = [&](int it) { return it == 1 || it % UPDATE == 0 || it == STEPS; };

    int it = sc.it;
    while (it < STEPS) {
        // run to the next diagnostic step (or one step when a signal must be served promptly)
        int nxt = it + 1;
        if (!is_diag(nxt)) {
            nxt = std::min(STEPS, (it / UPDATE + 1) * UPDATE);
            if (it < 1) nxt = 1;
            // poll signals at least every 64 steps
            nxt = std::min(nxt, it + 64);
        }
        rc = dns2d_step(s, nxt - it, nullptr, nullptr);
        if (rc) {
            die(s, rc, "dns2d_step");
            dns2d_destroy(s);
            return 1;
        }
        it = nxt;
        if (is_diag(it)) {
            float cflm = 0.0f;
            dns2d_next_dt(s, &cflm);
            dns2d_om2phys(s);
            double sigma = 0.0, pal = 0.0;
            dns2d_display_sigma(s, 2, &sigma);
            dns2d_get_scalars(s, &sc);
            if (ADAPT) {
                dns2d_palin(s, &pal);
                adapt_visc(sc, av, pal);
                dns2d_set_scalars(s, &sc);
            }
            append_row(rows, make_row(sc, pal, sigma, elapsed_active(), start_iter));
            std::printf(" ITERATION %6d T=%12.10f DT=%10.8f CN=%10.8f CFLM=%.6f Re=%12.5e VISC=%12.5e PALIN=%d SIG=%d "
                        "FPS=%.3f\n",
                        it, (double)sc.t, (double)sc.dt, (double)sc.cn, (double)sc.cflm, (double)sc.Re, (double)sc.visc,
                        rows.back().PALIN, rows.back().SIG, rows.back().FPS);
            if (MOV && it > 0 && it % UPDATE == 0) {
                char name[64];
                std::snprintf(name, sizeof(name), "omega_inferno_%05d.png", movie_frame + 1);
                if (!save_movie_frame(s, png, join(movie_folder, name), movie_F)) {
                    dns2d_destroy(s);
                    return 1;
                }
                ++movie_frame;
            }
            if (!steady_started && it >= warm) {
                dns2d_sync(s, 0);
                steady_begin = clk::now();
                steady_iter0 = it;
                steady_paused0 = paused;
                steady_started = true;
                std::printf("[BENCH] Steady FPS timer starts after iteration %d.\n", steady_iter0);
            }
        }
        if (g_pause_requested) {
            g_pause_requested = 0;
            g_resume_requested = 0;
            dns2d_sync(s, 0);
            const auto p0 = clk::now();
            std::printf("[SIGNAL] Received SIGUSR2; pausing at iteration %d. Send SIGCONT to resume.\n", it);
            std::fflush(stdout);
            while (!g_resume_requested && !g_exit_requested) std::this_thread::sleep_for(std::chrono::milliseconds(250));
            const double pe = std::chrono::duration<double>(clk::now() - p0).count();
            paused += pe;
            if (g_resume_requested) {
                g_resume_requested = 0;
                std::printf("[SIGNAL] Received SIGCONT; resuming after %.3f paused seconds.\n", pe);
                std::fflush(stdout);
            }
        }
        if (g_exit_requested) {
            interrupted = true;
            break;
        }
        if (g_save_restart_requested || g_save_requested) {
            const bool with_restart = g_save_restart_requested != 0;
            g_save_restart_requested = 0;
            g_save_requested = 0;
            dns2d_sync(s, 0);
            const double secs = elapsed_active();
            const double fps = secs > 0.0 ? (double)(it - start_iter) / secs : 0.0;
            dns2d_get_scalars(s, &sc);
            std::string folder = folder_name(sc, N, K0, Re, CFL);
            if (with_restart) {
                std::printf("[SIGNAL] Received SIGRTMIN; saving images and restart binary, then continuing.\n");
                folder += "_restart";
                if (!make_dir(folder)) return 1;
                const std::string rp = folder + "/restart.bin";
                if (dns2d_save_restart(s, rp.c_str())) {
                    std::fprintf(stderr, "saveRestartBin: %s\n", dns2d_last_error(s));
                    dns2d_destroy(s);
                    return 1;
                }
                std::printf("[SAVE] Wrote %s (restart binary)\n", rp.c_str());
            } else {
                std::printf("[SIGNAL] Received SIGUSR1; saving current state and continuing.\n");
            }
            dns2d_om2phys(s);
            double sigma = 0.0, pal = 0.0;
            dns2d_display_sigma(s, 2, &sigma);
            if (ADAPT) dns2d_palin(s, &pal);
            append_row(rows, make_row(sc, pal, sigma, secs, start_iter));
            if (!dump_outputs(s, rows, folder, UPDATE, secs, fps)) {
                dns2d_destroy(s);
                return 1;
            }
        }
    }

    dns2d_sync(s, 0);
    const auto tend = clk::now();
    const double elap = std::chrono::duration<double>(tend - tbegin).count() - paused;
    dns2d_get_scalars(s, &sc);
    const int done = sc.it - start_iter;
    const double fps = elap > 0.0 ? done / elap : 0.0;
    double steady_elap = 0.0, steady_fps = 0.0;
    const int steady_done = sc.it - steady_iter0;
    if (steady_started && steady_done > 0) {
        steady_elap = std::chrono::duration<double>(tend - steady_begin).count() - (paused - steady_paused0);
        steady_fps = steady_elap > 0.0 ? steady_done / steady_elap : 0.0;
    }
    std::printf(" Frames per second (FPS)            = %12.7f\n", fps);
    if (steady_started && steady_done > 0)
        std::printf(" Steady frames per second (FPS)     = %12.7f  (%d steps after warmup)\n", steady_fps, steady_done);
    std::printf(" Elapsed time (s): %12.7f\n", elap);
    std::printf(" FPS: %12.7f\n", fps);
    if (steady_started && steady_done > 0) {
        std::printf(" Steady elapsed time (s): %12.7f\n", steady_elap);
        std::printf(" Steady FPS: %12.7f\n", steady_fps);
    }
    std::printf(" Final T=%12.7f  CN=%12.7f  DT=%12.7f  VISC=%12.7f\n", (double)sc.t, (double)sc.cn, (double)sc.dt,
                (double)sc.visc);
    gpu_snapshot("end");
    if (phase_timing) {
        double ms[4];
        long long n[4];
        dns2d_phase_report(s, ms, n);
        const char *names[4] = {"row pass (STEP2A x-inverse + STEP2B products/x-forward)",
                                "column pass (STEP2B z-forward + STEP3 + STEP2A z-inverse)", "NEXTDT/CFLM",
                                "OM2PHYS + display sigma"};
        double tot = ms[0] + ms[1] + ms[2] + ms[3];
        std::printf("[PHASE] CUDA event timings for measured loop phases\n[PHASE] phase,total_ms,count,avg_ms,pct\n");
        for (int i = 0; i < 4; ++i)
            std::printf("[PHASE] %s,%.3f,%lld,%.3f,%.2f\n", names[i], ms[i], n[i], n[i] ? ms[i] / n[i] : 0.0,
                        tot > 0 ? 100.0 * ms[i] / tot : 0.0);
    }
    std::fflush(stdout);
    if (interrupted) {
        ignore_signals();
        const int sig = (int)g_exit_signal;
        if (!(sig == SIGHUP || sig == SIGTERM)) {
            std::printf("[SIGNAL] Received %s (%d); exiting without saving.\n", signal_name(sig), sig);
            dns2d_destroy(s);
            return 128 + sig;
        }
        std::printf("[SIGNAL] Received %s (%d); dumping current state before exit.\n", signal_name(sig), sig);
        dns2d_next_dt(s, nullptr);
        dns2d_om2phys(s);
        double sigma = 0.0, pal = 0.0;
        dns2d_display_sigma(s, 2, &sigma);
        if (ADAPT) dns2d_palin(s, &pal);
        dns2d_get_scalars(s, &sc);
        append_row(rows, make_row(sc, pal, sigma, elap, start_iter));
        const bool ok = dump_outputs(s, rows, folder_name(sc, N, K0, Re, CFL), UPDATE, elap, fps);
        dns2d_destroy(s);
        return ok ? 128 + sig : 1;
    }
    std::printf("[OUTPUT] Normal completion; no output files written.\n");
    dns2d_destroy(s);
    return 0;
}
