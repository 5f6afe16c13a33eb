// Output records of sea_ice_post (diagnostics_outputs.f90:1-189) and the
// file clean-up of clear_posts (diagnostics_ini_io.f90:1-100), written from a
// context's device state.
//
// The reference writes its outputs with list-directed WRITE (write(u,*)),
// whose layout is the compiler runtime's.  The reference builds with gfortran
// (godarCMakeFiles/gfortranFLAGS.cmake), so the layout here is libgfortran's
// list-directed output for default files: every record starts with a blank,
// items are separated by one blank, an INTEGER(4) is right-justified in 11
// columns and a REAL(8) is edited as G25.17E3 with scale factor 1 - F
// editing with 17 significant digits in 20 columns followed by 5 blanks when
// 0.1 <= |x| < 1e17 (and for zero), else 1PE25.17E3 - with the decimal digits
// correctly rounded (libgfortran takes them from the C library's printf, as
// this file does).  Records are not wrapped (gfortran's default record length
// for sequential formatted files is far above one record of n reals).
//
// Host code only.  The values come through the public read-out entry points,
// so this file sees the state exactly as a caller of godar_gpu_download does.
#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/godar_gpu.h"
#include "common.cuh"

#define TRY(expr)                        \
    do {                                 \
        int rc_ = (expr);                \
        if (rc_ != GODAR_OK) return rc_; \
    } while (0)

namespace godar {

// engine.cu: the context's floe count and the thread's last error message
int ctx_floe_count(const godar_ctx *c);
void set_last_error(const std::string &msg);

namespace {

void set_err(const std::string &msg) { set_last_error(msg); }

// One REAL(8) list-directed field (25 characters, no separator).
void g25_17(double x, char *out)
{
    char body[16];   // NaN or (-)Infinity
    if (std::isnan(x)) {
        std::snprintf(body, sizeof body, "NaN");
    } else if (std::isinf(x)) {
        std::snprintf(body, sizeof body, "%s", x < 0 ? "-Infinity" : "Infinity");
    } else {
        // 17 significant digits, correctly rounded: d.dddddddddddddddde[+-]xx
        char e[48];
        std::snprintf(e, sizeof e, "%.16e", x);
        const bool neg = e[0] == '-';
        const char *p = e + (neg ? 1 : 0);
        char dig[17];
        dig[0] = p[0];
        std::memcpy(dig + 1, p + 2, 16);
        const int e10 = std::atoi(p + 19);
        std::string s = neg ? "-" : "";
        if (x == 0.0) {
            s += "0.0000000000000000";
        } else if (e10 >= -1 && e10 <= 16) {
            // F editing: k integer digits, 17 - k decimals
            const int k = e10 + 1;
            if (k == 0) {
                s += "0.";
                s.append(dig, 17);
            } else {
                s.append(dig, k);
                s += '.';
                s.append(dig + k, 17 - k);
            }
        } else {
            s += dig[0];
            s += '.';
            s.append(dig + 1, 16);
            char ex[16];
            std::snprintf(ex, sizeof ex, "E%c%03d", e10 < 0 ? '-' : '+', e10 < 0 ? -e10 : e10);
            s += ex;
            std::snprintf(out, 26, "%25s", s.c_str());
            return;
        }
        // F editing: right-justified in w - (e + 2) = 20 columns, then the
        // e + 2 = 5 blanks where the exponent would be
        std::snprintf(out, 26, "%20s     ", s.c_str());
        return;
    }
    std::snprintf(out, 26, "%25s", body);
}

void put_real(std::string &rec, double x)
{
    char f[32];
    g25_17(x, f);
    rec += ' ';
    rec += f;
}

void put_int(std::string &rec, long long v)
{
    char f[32];
    std::snprintf(f, sizeof f, " %11lld", v);
    rec += f;
}

std::string path_of(const char *dir, const char *name, const char *expno)
{
    // "output/x." // trim(adjustl(expno_str))
    std::string e = expno ? expno : "";
    const size_t a = e.find_first_not_of(' ');
    const size_t b = e.find_last_not_of(' ');
    e = a == std::string::npos ? std::string() : e.substr(a, b - a + 1);
    return std::string(dir && *dir ? dir : "output") + "/" + name + "." + e;
}

int append(const std::string &path, const std::string &text)
{
    FILE *f = std::fopen(path.c_str(), "ab");
    if (!f) {
        set_err("cannot open " + path + ": " + std::strerror(errno));
        return GODAR_ERR_IO;
    }
    const size_t w = std::fwrite(text.data(), 1, text.size(), f);
    const int rc = std::fclose(f);
    if (w != text.size() || rc != 0) {
        set_err("cannot write " + path);
        return GODAR_ERR_IO;
    }
    return GODAR_OK;
}

// The 25 files of sea_ice_post in unit order (units 10-34) and the info file
// that clear_posts also removes.
const char *const kPerFloe[GODAR_F_COUNT] = {"x", "y", "u", "v", "r", "h", "theta", "omega",
                                             "tfx", "tfy", "fcx", "fcy", "fbx", "fby", "mom", "mc", "mb",
                                             "tsigxx", "tsigyy", "tsigxy", "tsigyx", "tp"};
const char *const kAll[] = {"x", "y", "u", "v", "r", "h", "theta", "omega", "bond",
                            "tfx", "tfy", "fcx", "fcy", "fbx", "fby", "mom", "mc", "mb",
                            "tsigxx", "tsigyy", "tsigxy", "tsigyx", "tp", "angle", "damage", "info"};

struct PairList {
    std::vector<int32_t> i, j;
    std::vector<double> v;
    std::vector<int> order;    // by (i, j): the reference's loop order
};

int read_pairs(godar_ctx *c, int which, PairList &L)
{
    int count = 0;
    TRY(godar_gpu_get_pairs(c, which, nullptr, nullptr, nullptr, 0, &count));
    L.i.resize(count); L.j.resize(count); L.v.resize(count);
    if (count > 0) {
        int got = 0;
        TRY(godar_gpu_get_pairs(c, which, L.i.data(), L.j.data(), L.v.data(), count, &got));
        if (got != count) { set_err("pair list changed while read"); return GODAR_ERR_STATE; }
    }
    L.order.resize(count);
    std::iota(L.order.begin(), L.order.end(), 0);
    std::sort(L.order.begin(), L.order.end(), [&](int a, int b) {
        return L.i[a] != L.i[b] ? L.i[a] < L.i[b] : L.j[a] < L.j[b];
    });
    return GODAR_OK;
}

}  // namespace

int posts_format_reals(const double *v, int n, char *out, size_t cap, size_t *len)
{
    std::string rec;
    rec.reserve((size_t)n * 26 + 1);
    for (int k = 0; k < n; k++) put_real(rec, v[k]);
    rec += '\n';
    if (len) *len = rec.size();
    if (!out) return GODAR_OK;
    if (cap < rec.size() + 1) { set_err("record does not fit"); return GODAR_ERR_CAPACITY; }
    std::memcpy(out, rec.c_str(), rec.size() + 1);
    return GODAR_OK;
}

int write_posts(godar_ctx *c, const char *dir, const char *expno, int tstep, double comp)
{
    const int n = ctx_floe_count(c);
    if (n <= 0) { set_err("no field"); return GODAR_ERR_STATE; }
    if (!(comp > 0)) { set_err("comp must be > 0"); return GODAR_ERR_BAD_INPUT; }
    std::vector<std::vector<double>> fl(GODAR_F_COUNT, std::vector<double>(n));
    std::vector<double *> ptr(GODAR_F_COUNT);
    for (int f = 0; f < GODAR_F_COUNT; f++) ptr[f] = fl[f].data();
    TRY(godar_gpu_download(c, ptr.data(), -1, nullptr, nullptr, nullptr, 0, nullptr));
    PairList bonds, cont;
    TRY(read_pairs(c, GODAR_P_BONDS, bonds));
    TRY(read_pairs(c, GODAR_P_CONTACTS, cont));
    const long long out_no = (long long)((double)tstep / comp);     // int(tstep / comp)
    const double pi = 4.0 * std::atan(1.0);                          // par_get.f90:35
    const double *x = fl[GODAR_F_X].data(), *y = fl[GODAR_F_Y].data();
    // bond (unit 18), damage (34): bond(j, i) == 1 in the loop i = 1..n,
    // j = 1..n (diagnostics_outputs.f90:155-166), the higher index first;
    // an empty record closes the bond file's block
    std::string rb, rd, ra;
    for (int q : bonds.order) {
        const int lo = bonds.i[q], hi = bonds.j[q];
        put_int(rb, out_no); put_int(rb, hi + 1); put_int(rb, lo + 1);
        rb += '\n';
        put_int(rd, out_no); put_int(rd, hi + 1); put_int(rd, lo + 1); put_real(rd, bonds.v[q]);
        rd += '\n';
    }
    rb += '\n';
    // angle (33): deltan(j, i) > 0, atan2(y(j) - y(i), x(j) - x(i)) * 180 / pi
    for (int q : cont.order) {
        const int lo = cont.i[q], hi = cont.j[q];
        if (!(cont.v[q] > 0.0)) continue;
        const double ang = (std::atan2(y[hi] - y[lo], x[hi] - x[lo]) * 180.0) / pi;
        put_int(ra, out_no); put_int(ra, hi + 1); put_int(ra, lo + 1); put_real(ra, ang);
        ra += '\n';
    }
    // the per-floe records are formatted on host threads (about 0.3 us per
    // value), then appended in unit order
    std::vector<std::string> recs(GODAR_F_COUNT);
    {
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const int T = (int)std::min<unsigned>(hw, GODAR_F_COUNT);
        std::atomic<int> next{0};
        auto work = [&] {
            for (int f; (f = next.fetch_add(1)) < GODAR_F_COUNT;) {
                std::string &rec = recs[f];
                rec.reserve((size_t)n * 26 + 1);
                for (int k = 0; k < n; k++) put_real(rec, fl[f][k]);
                rec += '\n';
            }
        };
        std::vector<std::thread> th;
        for (int w = 1; w < T; w++) th.emplace_back(work);
        work();
        for (auto &t : th) t.join();
    }
    for (int f = 0; f < GODAR_F_COUNT; f++) TRY(append(path_of(dir, kPerFloe[f], expno), recs[f]));
    TRY(append(path_of(dir, "bond", expno), rb));
    TRY(append(path_of(dir, "angle", expno), ra));
    TRY(append(path_of(dir, "damage", expno), rd));
    return GODAR_OK;
}

int clear_posts(const char *dir, const char *expno)
{
    for (const char *name : kAll) {
        const std::string p = path_of(dir, name, expno);
        if (std::remove(p.c_str()) != 0 && errno != ENOENT) {
            set_err("cannot delete " + p + ": " + std::strerror(errno));
            return GODAR_ERR_IO;
        }
    }
    return GODAR_OK;
}

}  // namespace godar

extern "C" {

int godar_gpu_write_posts(godar_ctx *ctx, const char *dir, const char *expno, int tstep, double comp)
{
    if (!ctx || !expno) return GODAR_ERR_BAD_INPUT;
    return godar::write_posts(ctx, dir, expno, tstep, comp);
}

int godar_gpu_clear_posts(const char *dir, const char *expno)
{
    if (!expno) return GODAR_ERR_BAD_INPUT;
    return godar::clear_posts(dir, expno);
}

int godar_posts_format_reals(const double *v, int n, char *out, size_t cap, size_t *len)
{
    if ((!v && n > 0) || n < 0) return GODAR_ERR_BAD_INPUT;
    return godar::posts_format_reals(v, n, out, cap, len);
}

}  // extern "C"
