// Host engine and C ABI of libgodar_gpu.so.
//
// An Engine holds one batch of floe fields ("instances") laid out back to back
// in structure-of-arrays device buffers (see common.cuh).  It replaces the
// state set-up of ini_get/broadcasting_ini (ini_get.f90:1-249,
// mpi_coms.f90:1-218), the time loop's `call stepper` (godar.f90:191-193) and
// the reads of the output step (diagnostics_outputs.f90:149-182).
//
// Host-side control flow of a step call: time steps run in chunks of device
// launches; after each chunk the host reads the status word.  A floe that
// moved more than half the neighbour-list skin freezes the batch after that
// (still valid) step; the host then rebuilds the rows (kernel a) and runs the
// remaining steps.  Batch membership changes (admission, removal) are applied
// between step calls by a synchronous "commit" that re-lays the buffers and
// carries every existing instance's floe, pair and bond state over.
#include <algorithm>
#include <array>
#include <map>
#include <tuple>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstddef>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/godar_gpu.h"
#include "common.cuh"
#include "detmath.cuh"
#include "kernels.h"

using namespace godar;

namespace {

thread_local std::string g_last_error;

void set_err(const char *msg) { g_last_error = msg; }

#define CK(call)                                                                 \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess) {                                                 \
            g_last_error = std::string(#call) + ": " + cudaGetErrorString(e_);   \
            return GODAR_ERR_CUDA;                                               \
        }                                                                        \
    } while (0)

#define TRY(expr)                   \
    do {                            \
        int rc_ = (expr);           \
        if (rc_ != GODAR_OK) return rc_; \
    } while (0)

// ------------------------------------------------------------ device buffers
// A stream-ordered memory pool that keeps what is freed (release threshold
// at its maximum): once a batch has reached its working size, buffer growth
// and relayouts are served from memory the pool already holds.  cudaMalloc
// and cudaFree take about a millisecond each, stall for up to a hundred on a
// busy machine, and cudaFree waits for the device.
struct Pool {
    cudaMemPool_t pool = nullptr;
    cudaStream_t st = nullptr;      // allocations are ordered on this stream
};

struct Buf {
    void *p = nullptr;
    size_t bytes = 0;
    bool pooled = false;
    Buf() = default;
    Buf(const Buf &) = delete;
    Buf &operator=(const Buf &) = delete;
    ~Buf() { free_mem(); }
    void free_mem() {
        if (!p) return;
        if (pooled) {
            // whatever any stream still does with the buffer ends first, and
            // the memory is back in the pool before the call returns
            cudaDeviceSynchronize();
            cudaFreeAsync(p, nullptr);
            cudaStreamSynchronize(nullptr);
        } else {
            cudaFree(p);
        }
        p = nullptr;
    }
    // A buffer that has to grow again grows by at least half its size, so a
    // batch whose membership keeps changing reallocates rarely.
    int ensure(size_t b, std::atomic<size_t> *acct, const Pool *pl = nullptr) {
        if (b <= bytes && p) return GODAR_OK;
        const size_t grown = p ? std::max(b, bytes + bytes / 2) : b;
        if (p) { free_mem(); if (acct) *acct -= bytes; bytes = 0; }
        size_t nb = std::max<size_t>(grown, 256);
        pooled = pl && pl->pool;
        cudaError_t e = pooled ? cudaMallocFromPoolAsync(&p, nb, pl->pool, pl->st) : cudaMalloc(&p, nb);
        if (e != cudaSuccess) { g_last_error = std::string("device allocation: ") + cudaGetErrorString(e); p = nullptr; return GODAR_ERR_NOMEM; }
        bytes = nb;
        if (acct) *acct += bytes;
        return GODAR_OK;
    }
    void release(std::atomic<size_t> *acct) { if (p) { free_mem(); if (acct) *acct -= bytes; } p = nullptr; bytes = 0; }
    template <class T> T *as() const { return (T *)p; }
};

inline int ilog2ceil(uint64_t v) { int b = 0; while ((1ULL << b) < v) b++; return b; }

// ------------------------------------------------------------ instances
struct HostBonds {           // one instance's bond table, id order
    std::vector<int> off;    // n+1
    std::vector<int> hi;
    std::vector<double> rb, hb, lb, sb, ib, dnb, dtb, thji, thij, dmg;
    std::vector<int> flag;
};

// State a checkpoint restores beyond the floe state: wall histories, the
// complete bond table, and the pair histories (by reference ids).
struct RestoreExtra {
    std::vector<double> dtb1, dtb2, thb1, thb2;
    HostBonds bonds;
    std::vector<int> hi, hj;
    std::vector<double> h4;
};

// Checkpoint layout (host byte order): this header; 12 arrays of n doubles
// (x y u v r h theta omega deltat_bc1 deltat_bc2 theta_bc1 theta_bc2, by
// reference index); nb bonds, each int32 {i, j, flag, 0} then doubles
// {rb hb lb sb ib deltanb deltatb thetarelb(j,i) thetarelb(i,j) damageb},
// ordered by i then j (i < j); nh pair histories, each int32 {i, j} then
// doubles {deltat thetarelc fcn fct}, ordered by i then j.
struct CkptHeader {
    char magic[8];
    int32_t version, precision, n, nb, nh, pad;
};

struct Inst {
    int handle = -1;
    godar_params prm{};
    int n = 0;
    int off = 0;
    long long steps = 0;
    std::vector<double> field;   // 4*fnx*fny or empty
    // host copy of the initial state until the first commit
    bool pending = false;        // not yet on the device
    bool fresh = false;          // create bonds at commit (time step 1, not a restart)
    std::vector<double> x, y, r, h, th, om, u, v;
    std::vector<int> bi, bj;
    std::vector<double> dmg;
    // bonds on the device (count and first index in the batch table)
    int nb = 0, boff = 0;
    double rmax = 0.0;
    std::shared_ptr<RestoreExtra> rx;   // set when the instance comes from a checkpoint
};

double wrapd_host(double d, double L, bool per)
{
    if (!per) return d;
    if (d > 0.5 * L) d = d - L;
    else if (d < -0.5 * L) d = d + L;
    return d;
}

// bond_properties (bonds.f90:237-269) for pair (i,j) at distance dist
void bond_geom(const godar_params &p, double ri, double rj, double hi, double hj, double dist,
               double &rb, double &hb, double &lb, double &sb, double &ib)
{
    rb = p.lambda_rb * (ri < rj ? ri : rj);
    hb = (hi + hj) / 2.0;
    lb = dist;
    sb = (2.0 * rb) * hb;
    ib = ((2.0 / 3.0) * hb) * ((rb * rb) * rb);
}

// restart bonds given as (i, j, damage) lists (read_sparse_restart,
// ini_get.f90:252-311); geometry from the uploaded positions.
void restart_bonds(const Inst &I, HostBonds &B)
{
    const godar_params &p = I.prm;
    const int n = I.n;
    const bool px = p.boundary & GODAR_BC_PERIODIC_X, py = p.boundary & GODAR_BC_PERIODIC_Y;
    std::vector<std::vector<std::pair<int, double>>> part(n);
    for (size_t k = 0; k < I.bi.size(); k++) {
        int i = I.bi[k], j = I.bj[k];
        if (i > j) std::swap(i, j);
        part[i].push_back({j, I.dmg.empty() ? 0.0 : I.dmg[k]});
    }
    B.off.assign(n + 1, 0);
    for (int i = 0; i < n; i++) {
        std::sort(part[i].begin(), part[i].end());
        part[i].erase(std::unique(part[i].begin(), part[i].end(),
                                  [](auto &a, auto &b) { return a.first == b.first; }), part[i].end());
        B.off[i + 1] = B.off[i] + (int)part[i].size();
    }
    const int nb = B.off[n];
    auto rs = [&](std::vector<double> &v) { v.assign(nb, 0.0); };
    B.hi.assign(nb, 0); B.flag.assign(nb, 1);
    rs(B.rb); rs(B.hb); rs(B.lb); rs(B.sb); rs(B.ib); rs(B.dnb); rs(B.dtb); rs(B.thji); rs(B.thij); rs(B.dmg);
    for (int i = 0; i < n; i++)
        for (size_t k = 0; k < part[i].size(); k++) {
            const int j = part[i][k].first, q = B.off[i] + (int)k;
            const double dx = wrapd_host(I.x[i] - I.x[j], p.nx, px);
            const double dy = wrapd_host(I.y[i] - I.y[j], p.ny, py);
            const double dist = std::sqrt(dx * dx + dy * dy);
            B.hi[q] = j;
            B.dmg[q] = part[i][k].second;
            bond_geom(p, I.r[i], I.r[j], I.h[i], I.h[j], dist, B.rb[q], B.hb[q], B.lb[q], B.sb[q], B.ib[q]);
        }
}

}  // namespace

// ====================================================================== Engine
struct PoolOwner {
    Pool mp;
    ~PoolOwner() { if (mp.pool) cudaMemPoolDestroy(mp.pool); }
};

struct Engine {
    // first member, so that it is destroyed after every buffer drawn from it
    PoolOwner po;
    Pool &mp = po.mp;
    int prec = GODAR_PREC_FP64;
    size_t budget = 0;
    cudaStream_t st = nullptr;
    // second stream: the bond kernel runs beside the pair kernels when no
    // field of the batch has ridging (a ridging event tells the bond kernel
    // the pair's new radius, which orders the two)
    cudaStream_t st2 = nullptr;
    // read-back: godar_batch_get_all_async gathers a step's results on stg
    // into one of two staging slots and copies them to the host on stc while
    // the next steps compute; two read-backs can be in flight, so that the
    // copies run back to back
    cudaStream_t stc = nullptr, stg = nullptr;
    cudaEvent_t ev_state = nullptr;
    cudaEvent_t ev_gath[2] = {nullptr, nullptr}, ev_copy[2] = {nullptr, nullptr};
    bool copy_pend[2] = {false, false};   // the host has not waited for the slot's copy
    bool gath_rec[2] = {false, false};    // the slot's gather event has been recorded
    int gath_side[2] = {0, 0};            // the side the slot's gather read
    int aslot = 0;                        // the slot of the next read-back
    static constexpr int MAX_ASYNC_FIELDS = 4;
    Buf async_tmp[2][MAX_ASYNC_FIELDS];
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool ridging_any = false;
    // mixed path: the bond kernel works on copies of the dynamic records in
    // its own order; the bond table is brought up to date before anything
    // else reads it
    bool wdirty = false;
    // the last step of every call computes the diagnostics (per-floe forces,
    // stresses, contact list, counters); a caller that only reads the state
    // can switch them off
    bool diagnostics = true;
    int wnb = 0;
    // off by default: the overlap gains about 2% of a step on the benchmark
    // ensemble, and kernels sharing the GPU make per-kernel times meaningless
    bool overlap_bonds = false;
    bool walls_any = false;        // some field of the batch has a solid wall

    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::atomic<size_t> bytes{0};
    std::vector<Inst> insts;      // committed + pending, layout order
    int next_handle = 0;
    bool dirty = false;           // membership changed since the last commit
    int N = 0, NB = 0;
    long long E = 0;              // rows in use
    long long Ecap = 0;
    long long C = 0;              // cells
    int cur = 0;
    bool have_rows = false;
    int chunk = 16;
    int block = 128;
    double last_ms = 0.0;
    double accum_ms = 0.0;
    bool timing_open = false;
    unsigned long long counters[4] = {0, 0, 0, 0};
    // Verlet skin = max(1 m, skin_frac (r_max + rtree)); a rebuild costs
    // about 25 ms on 2.2M floes, and 1% keeps rebuilds hundreds to thousands
    // of steps apart on the benchmark fields while shortening the rows
    // (GODAR_SKIN_FRAC overrides it; no result depends on it)
    double skin_frac = 0.01;
    double kernel_ms = 0.0;        // device time inside step kernels
    long long launches = 0;        // time steps launched
    // the kernels of a time step: mixed [pair screen, pair work list, bonds,
    // floe sums, floe update]; FP64 [entry screen, general work list, bond
    // work list, row sums, floe update]
    static constexpr int NPH = 5;
    static constexpr int NEV = NPH + 2;   // timing events per step
    double phase_ms[NPH] = {0, 0, 0, 0, 0};
    long long kernel_launches = 0;   // step kernels launched
    // launch configuration of each kernel: block size in the low 16 bits,
    // kernel variant above (the screen's items per lane: 0 = 8, 1 = 4,
    // 2 = 16; the bonds: 1 = records streamed through shared memory by bulk
    // copies)
    int blk[NPH] = {128, 128, 128, 128, 128};
    static int cfg_block(int c) { return c & 0xffff; }
    static int cfg_variant(int c) { return c >> 16; }
    // online autotuner: neither block sizes nor variants change a result
    // (every output is per entry, per bond or per floe in a fixed order), so
    // the first steps of a batch try each kernel's candidates in turn and
    // keep the fastest
    static constexpr int MAXCFG = 9;
    static constexpr int TUNE_ROUNDS = 2;    // samples of each candidate
    static constexpr int PDL_MAX_FLOES = 148 * 1024;
    int cfg[NPH][MAXCFG] = {};
    int ncfg[NPH] = {};
    double tune_ms[NPH][MAXCFG] = {};
    int tune_n[NPH][MAXCFG] = {};
    int tune_left = 0;               // tuning steps still to run
    int tune_step = 0;               // candidate rotation across calls
    int tuned_n = 0;                 // batch size the blocks were tuned for
    bool tune_on = true;
    bool tune_log = false;           // GODAR_TUNE_LOG=1: print the tuner's measurements
    // GODAR_TEST_WAIT_SPINS=n (tests of the timeout path only): the bulk-copy
    // bond kernel first waits at most n tries on a barrier that nothing
    // completes, so that its step returns GODAR_ERR_TIMEOUT
    unsigned test_wait_spins = 0;
    // CUDA graphs of whole chunks of steps, keyed by (steps, start side,
    // diagnostics on the last step); invalid after every rebuild
    bool graphs_on = true;
    // run() brackets the kernels of every phase_every-th step of a chunk with
    // CUDA events (0: none; the autotuner's steps always are).  An event
    // record between two kernels of a captured graph costs several
    // microseconds of device time, so steps are sampled, and by default not
    // timed at all.
    int phase_every = 0;
    long long phase_steps = 0;       // steps whose kernels were timed
    long long graph_gen = -1;
    // captured chunks by (steps, first side, diagnostics on the last step | 2 x
    // the interval of the steps whose kernels record timing events)
    std::map<std::tuple<int, int, int>, cudaGraphExec_t> graphs;
    std::map<std::tuple<int, int, int>, int> graph_uses;   // direct launches per key in this generation
    long long graph_launches = 0;
    long long rebuilds = 0;        // neighbour-list rebuilds
    double rebuild_ms = 0.0;       // their host wall time
    std::vector<cudaEvent_t> kev;  // per-launch events of a chunk
    std::vector<InstParams> hparams;

    // floe state (two sides) and bond table, each in a set that a batch
    // relayout replaces as a whole
    struct FloeSet {
        Buf x[2], y[2], th[2], u[2], v[2], om[2], r[2], h[2], dtb1[2], dtb2[2], thb1[2], thb2[2];
        Buf id[2], x0[2], y0[2], snap[2];
    };
    struct BondSet {
        Buf bond_off, bond_hi, bstat, bdyn[1];   // bond state, updated in place
    };
    std::unique_ptr<FloeSet> F = std::make_unique<FloeSet>();
    std::unique_ptr<BondSet> BS = std::make_unique<BondSet>();
    // the sets of the previous layout, the target of the next commit
    std::unique_ptr<FloeSet> spareF;
    std::unique_ptr<BondSet> spareB;
    // commit scratch: old slot of every new slot, old index of every new
    // bond, per-instance offset tables
    Buf repack_b, small_b, bmap_b, rule_b;
    Buf inst_b, params_b, field_b;
    // rows (primary) and rebuild scratch (secondary)
    Buf up_off, lo_off, ent_up, ent_lo, bidx, hist[1], edist, pdn;
    // mixed path: row of every owner entry, partner index, flags, pair records;
    // bond records, bond slots and the partner-bond lists
    Buf erow_up, lo_of, pfl, lfl, prec_b, prx_b, pdg_b, work_b, work_st_b, nwork_b, fsum_b, frex_b, fdg_b, clist_b, cscan_b;
    // FP64 path: the pair records and the bond work list (the row of every
    // owner entry, the pair flags and the general work list are the mixed
    // path's erow_up, pfl and work_b)
    Buf frec_b, fwork1_b;
    // FP64 path, per rebuild: the pairs that can act on a plain step before
    // the next rebuild (a byte per pair), their count at the head of every
    // row (owner, partner), and the list of their owner-row positions
    Buf flisted_b, fupn_b, flon_b, fpart_b, fpos_b, fplist_b;
    long long Lc = 0;
    long long Ec = 0;             // mixed path: owner entries on the contact list
    Buf brec, bdg, bsp, bst32, bflag_b, wdyn_b, wsp_b, winv_b, perm_b, wfo_b, bfo, slot_of, blo_start, blo_end, bkeys, bvals, bkeys_alt, bvals_alt, brs_counts, bscan;
    Buf row_off2, nlo2, ent2, dist2, cnt, old_slot;
    Buf up_off2, lo_off2, nup, ent_up2, ent_lo2, bidx2, hist2;
    Buf keys, vals, keys_alt, vals_alt, rs_counts, scan_scratch, cstart, cend;
    // mixed path: the screening's displacement bound (see k_pairs_screen)
    Buf dsp_b;
    // outputs and status
    // status: two ints, the status word and the global number of the first
    // step that expired (INT_MAX: none), read back together after each chunk
    Buf diag, status, counters_b, tmp_out, tmp_i, tmp_j, tmp_v, tmp_cnt;
    // pinned status mirror
    int *h_status = nullptr;
    // the global number of the next step to launch, counted from the last
    // rebuild; kernels read the running chunk's first one from step_base_b
    int gbase = 0;
    Buf step_base_b;
    // asynchronous steps (godar_batch_step_async): chunks launched whose
    // status has not been read yet, oldest first.  Each has a pinned slot
    // that receives the status word and the first expired step after it.
    struct Pending {
        int base, K, c0, slot;
        bool diag;                 // its last step produced the diagnostics
        std::vector<double> uvw;   // the uniform forcing it ran with (empty: as admitted)
    };
    static constexpr int RING = 16;
    std::deque<Pending> pend;
    int *h_ring = nullptr;
    cudaEvent_t ring_ev[RING] = {};
    int ring_next = 0;
    std::vector<double> cur_uvw;   // the last uniform forcing set since the last relayout
    // pinned copies of the uniform forcing for its queued uploads (a copy
    // from pageable memory may wait for the stream)
    static constexpr int FRING = 4;
    double *fring[FRING] = {};
    size_t fring_cap = 0;          // doubles per buffer
    cudaEvent_t fring_ev[FRING] = {};
    bool fring_used[FRING] = {};
    int fring_next = 0;

    size_t hist_elem() const { return prec == GODAR_PREC_FP64 ? sizeof(Hist4<double>) : sizeof(Hist4<float>); }

    ~Engine() {
        if (stc) cudaStreamSynchronize(stc);
        if (stg) cudaStreamSynchronize(stg);
        if (st) cudaStreamSynchronize(st);
        drop_graphs();
        for (auto e : kev) cudaEventDestroy(e);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (h_status) cudaFreeHost(h_status);
        if (h_ring) cudaFreeHost(h_ring);
        for (auto e : ring_ev)
            if (e) cudaEventDestroy(e);
        for (int q = 0; q < FRING; q++) {
            if (fring[q]) cudaFreeHost(fring[q]);
            if (fring_ev[q]) cudaEventDestroy(fring_ev[q]);
        }
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (st2) cudaStreamDestroy(st2);
        if (stc) cudaStreamDestroy(stc);
        if (stg) cudaStreamDestroy(stg);
        for (int q = 0; q < 2; q++) {
            if (ev_gath[q]) cudaEventDestroy(ev_gath[q]);
            if (ev_copy[q]) cudaEventDestroy(ev_copy[q]);
        }
        if (ev_state) cudaEventDestroy(ev_state);
        if (st) cudaStreamDestroy(st);
    }

    int init(int precision, size_t bud) {
        prec = precision;
        budget = bud;
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
            cudaGetLastError();
            set_err("no CUDA device visible");
            return GODAR_ERR_NO_DEVICE;
        }
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&stc, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&stg, cudaStreamNonBlocking));
        for (int q = 0; q < 2; q++) {
            CK(cudaEventCreateWithFlags(&ev_gath[q], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&ev_copy[q], cudaEventDisableTiming));
        }
        {
            int dev = 0, pools = 0;
            CK(cudaGetDevice(&dev));
            cudaDeviceGetAttribute(&pools, cudaDevAttrMemoryPoolsSupported, dev);
            if (pools) {
                cudaMemPoolProps pp = {};
                pp.allocType = cudaMemAllocationTypePinned;
                pp.location.type = cudaMemLocationTypeDevice;
                pp.location.id = dev;
                CK(cudaMemPoolCreate(&mp.pool, &pp));
                unsigned long long keep = ~0ULL;
                CK(cudaMemPoolSetAttribute(mp.pool, cudaMemPoolAttrReleaseThreshold, &keep));
                mp.st = st;
            }
            cudaGetLastError();
        }
        CK(cudaEventCreateWithFlags(&ev_state, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
        CK(cudaEventCreate(&ev0));
        CK(cudaEventCreate(&ev1));
        CK(cudaMallocHost(&h_status, 4 * sizeof(int)));
        CK(cudaMallocHost(&h_ring, RING * 4 * sizeof(int)));
        for (auto &e : ring_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        for (auto &e : fring_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        TRY(step_base_b.ensure(sizeof(int), &bytes, &mp));
        CK(cudaMemsetAsync(step_base_b.p, 0, sizeof(int), st));
        TRY(status.ensure(2 * sizeof(int), &bytes, &mp));
        TRY(counters_b.ensure(4 * sizeof(unsigned long long), &bytes, &mp));
        TRY(tmp_cnt.ensure(sizeof(int), &bytes, &mp));
        TRY(dsp_b.ensure(4 * sizeof(unsigned), &bytes, &mp));
        CK(cudaMemsetAsync(dsp_b.p, 0, 4 * sizeof(unsigned), st));
        TRY(reset_status());
        const char *sk = getenv("GODAR_SKIN_FRAC");
        if (sk) skin_frac = atof(sk);
        const char *ch = getenv("GODAR_CHUNK");
        if (ch) chunk = std::max(1, atoi(ch));
        const char *bl = getenv("GODAR_BLOCK");
        if (bl) block = std::max(32, atoi(bl));
        if (prec == GODAR_PREC_FP64) {
            // five kernels: the screen (phase 0), the pair physics of the
            // general and the bond work lists (phases 1, 2), the row sums
            // (phase 3) and the floe update (phase 4); all but the screen at
            // most 128 threads per block
            // the screen: every block size with 2, 1 and 4 entries per lane
            for (int v = 0; v < 3; v++)
                for (int k = 0; k < 3; k++) cfg[0][3 * v + k] = (64 << k) | (v << 16);
            ncfg[0] = 9;
            for (int q = 1; q < NPH; q++) { ncfg[q] = 3; cfg[q][0] = 32; cfg[q][1] = 64; cfg[q][2] = 128; }
        } else {
            for (int q = 0; q < NPH; q++) {
                ncfg[q] = 3;
                cfg[q][0] = 64; cfg[q][1] = 128; cfg[q][2] = 256;
            }
            // the screen: every block size with 8, 4 and 16 items per lane
            for (int v = 0; v < 3; v++)
                for (int k = 0; k < 3; k++) cfg[0][3 * v + k] = (64 << k) | (v << 16);
            ncfg[0] = 9;
            // the bonds: one lane per bond at three block sizes, or tiles of
            // 128 streamed through shared memory
            cfg[2][3] = 128 | (1 << 16);
            ncfg[2] = 4;
        }
        if (bl)
            for (int q = 0; q < NPH; q++) blk[q] = std::min(std::max(32, atoi(bl) & ~31), prec == GODAR_PREC_FP64 && q > 0 ? 128 : 256);
        // GODAR_BOND_VARIANT: the mixed bond kernel's variant, fixed (the
        // tuner keeps choosing the other kernels' configurations)
        const char *bv = getenv("GODAR_BOND_VARIANT");
        if (bv && prec != GODAR_PREC_FP64) {
            const int v = std::min(std::max(0, atoi(bv)), 1);
            blk[2] = (v ? 128 : cfg_block(blk[2])) | (v << 16);
            cfg[2][0] = blk[2];
            ncfg[2] = 1;
        }
        const char *tu = getenv("GODAR_TUNE");
        if (tu) tune_on = atoi(tu) != 0;
        const char *tl = getenv("GODAR_TUNE_LOG");
        if (tl) tune_log = atoi(tl) != 0;
        const char *tw = getenv("GODAR_TEST_WAIT_SPINS");
        if (tw) test_wait_spins = (unsigned)std::max(0, atoi(tw));
        if (bl) tune_on = false;
        const char *ob = getenv("GODAR_OVERLAP_BONDS");
        if (ob) overlap_bonds = atoi(ob) != 0;
        const char *gr = getenv("GODAR_GRAPHS");
        if (gr) graphs_on = atoi(gr) != 0;

        return GODAR_OK;
    }

    Views make_views(const FloeSet &f, const BondSet &b) const {
        Views V{};
        V.N = N;
        V.ninst = (int)insts.size();
        V.P = params_b.as<InstParams>();
        V.inst = inst_b.as<int>();
        for (int s = 0; s < 2; s++) {
            V.x[s] = f.x[s].as<double>(); V.y[s] = f.y[s].as<double>(); V.th[s] = f.th[s].as<double>();
            V.u[s] = f.u[s].as<double>(); V.v[s] = f.v[s].as<double>(); V.om[s] = f.om[s].as<double>();
            V.r[s] = f.r[s].as<double>(); V.h[s] = f.h[s].as<double>();
            V.dtb1[s] = f.dtb1[s].as<double>(); V.dtb2[s] = f.dtb2[s].as<double>();
            V.thb1[s] = f.thb1[s].as<double>(); V.thb2[s] = f.thb2[s].as<double>();
            V.id[s] = f.id[s].as<int>(); V.x0[s] = f.x0[s].as<double>(); V.y0[s] = f.y0[s].as<double>();
            V.snap[s] = f.snap[s].as<Snap>();
            // pair histories and bonds are updated in place (one thread owns
            // a pair or a bond in a step): both sides are the one table
            V.hist[s] = hist[0].p;
            V.bdyn[s] = b.bdyn[0].as<BondDyn>();
        }
        V.up_off = up_off.as<int>(); V.lo_off = lo_off.as<int>();
        V.ent_up = ent_up.as<int2>(); V.ent_lo = ent_lo.as<int2>();
        V.bidx = bidx.as<int>(); V.edist = edist.as<double>(); V.pdn = pdn.as<float>();
        V.bond_off = b.bond_off.as<int>(); V.bond_hi = b.bond_hi.as<int>();
        V.bstat = b.bstat.as<BondStat>();
        V.field = field_b.as<double>();
        V.diag = diag.as<double>();
        V.status = status.as<int>(); V.expired_at = status.as<int>() + 1;
        V.step_base = step_base_b.as<int>();
        V.counters = counters_b.as<unsigned long long>();
        return V;
    }

    Views views() const { return make_views(*F, *BS); }

    // No error and no expiry: status word 0, first expired step INT_MAX.
    int reset_status() {
        const int init[2] = {0, INT_MAX};
        CK(cudaMemcpyAsync(status.p, init, sizeof(init), cudaMemcpyHostToDevice, st));
        return GODAR_OK;
    }

    Inst *find(int handle) {
        for (auto &I : insts) if (I.handle == handle) return &I;
        return nullptr;
    }

    static size_t instance_bytes(int n, int nb, int precision) {
        // floe state (two sides, snapshots, ids, rebuild origins) and about 12
        // neighbour-superset pairs per floe: owner and partner rows, history,
        // and the rebuild's second generation; the mixed path adds the window
        // partials and the partners' shares; floe and bond sets count twice,
        // for the previous layout kept as the next commit's target
        const bool fp64 = precision == GODAR_PREC_FP64;
        const size_t per_pair = fp64 ? (8 + 8 + 4 + 32 + 8 + 4 + 4 + 1 + 2 * 32 + 1 + 16 + 4 + FP64_PAIR_REC_BYTES) + (16 + 16 + 8 + 8 + 4 + 32)
                                     : (8 + 8 + 4 + 16 + 4 + 4 + 4 + 1 + 1 + 32 + 8 + 32) +
                                           (16 + 16 + 8 + 8 + 4 + 16);
        const size_t per_floe = 2 * (2 * 15 * 8 + 2 * 48) + 64 + 12 * per_pair + (fp64 ? 8 * FP64_FLOE_SUMS : 12 + 68);
        const size_t per_bond = 2 * (4 + sizeof(BondStat) + sizeof(BondDyn)) + 8 +
                                (fp64 ? 0 : 32 + 64 + 8 + 8 + 16 + 32 + 2);
        return (size_t)n * per_floe + (size_t)nb * per_bond + 4096;
    }

    // bonds of a field not yet on the device: its restart list, or an upper
    // estimate of four per floe for a fresh field with cohesion
    static int bond_estimate(int n, int nrestart, bool fresh, bool cohesion) {
        return nrestart > 0 ? nrestart : (fresh && cohesion ? 4 * n : 0);
    }

    size_t committed_bytes() const {
        size_t s = 0;
        for (auto &I : insts)
            s += instance_bytes(I.n, I.pending ? bond_estimate(I.n, (int)I.bi.size(), I.fresh, I.prm.cohesion) : I.nb, prec);
        return s;
    }

    // -------------------------------------------------------------- admission
    int add(const godar_params *p, int n, const double *xx, const double *yy, const double *rr,
            const double *hh, const double *tt, const double *oo, const double *uu, const double *vv,
            int nbr, const int32_t *bi, const int32_t *bj, const double *dm_, const double *fld,
            int fresh, int *out_handle) {
        if (!p || n <= 0 || !xx || !yy || !rr || !hh) { set_err("null input or n <= 0"); return GODAR_ERR_BAD_INPUT; }
        if (nbr > 0 && (!bi || !bj)) { set_err("bond lists missing"); return GODAR_ERR_BAD_INPUT; }
        if (!(p->dt > 0) || !(p->nx > 0) || !(p->ny > 0) || !(p->rtree >= 0)) { set_err("bad dt/nx/ny/rtree"); return GODAR_ERR_BAD_INPUT; }
        if (p->field_nx || p->field_ny) {
            if (p->field_nx < 2 || p->field_ny < 2 || !fld) { set_err("forcing grid needs >= 2x2 nodes and data"); return GODAR_ERR_BAD_INPUT; }
        }
        if (budget) {
            size_t need = instance_bytes(n, bond_estimate(n, nbr, fresh != 0, p->cohesion != 0), prec);
            if (committed_bytes() + need > budget) { set_err("HBM budget exceeded"); return GODAR_ERR_BUDGET; }
        }
        Inst I;
        I.handle = next_handle++;
        I.prm = *p;
        I.n = n;
        I.pending = true;
        I.fresh = fresh != 0;
        auto cp = [n](const double *a, std::vector<double> &dst) {
            if (a) dst.assign(a, a + n); else dst.assign(n, 0.0);
        };
        cp(xx, I.x); cp(yy, I.y); cp(rr, I.r); cp(hh, I.h); cp(tt, I.th); cp(oo, I.om); cp(uu, I.u); cp(vv, I.v);
        for (int i = 0; i < n; i++) {
            if (!std::isfinite(I.x[i]) || !std::isfinite(I.y[i]) || !(I.r[i] > 0) || !(I.h[i] > 0) ||
                !std::isfinite(I.th[i]) || !std::isfinite(I.om[i]) || !std::isfinite(I.u[i]) || !std::isfinite(I.v[i])) {
                set_err("non-finite floe state or non-positive radius/thickness");
                return GODAR_ERR_BAD_INPUT;
            }
            I.rmax = std::max(I.rmax, I.r[i]);
        }
        for (int k = 0; k < nbr; k++) {
            if (bi[k] < 0 || bi[k] >= n || bj[k] < 0 || bj[k] >= n || bi[k] == bj[k]) { set_err("bad bond index"); return GODAR_ERR_BAD_INPUT; }
            I.bi.push_back(bi[k]); I.bj.push_back(bj[k]);
            I.dmg.push_back(dm_ ? dm_[k] : 0.0);
        }
        if (fld) I.field.assign(fld, fld + (size_t)4 * p->field_nx * p->field_ny);
        const double Rmax = I.rmax + p->rtree + skin_of(I);
        if ((p->boundary & GODAR_BC_PERIODIC_X) && p->nx < 2.0 * Rmax) { set_err("periodic x needs nx >= 2 (r_max + rtree + skin)"); return GODAR_ERR_BAD_INPUT; }
        if ((p->boundary & GODAR_BC_PERIODIC_Y) && p->ny < 2.0 * Rmax) { set_err("periodic y needs ny >= 2 (r_max + rtree + skin)"); return GODAR_ERR_BAD_INPUT; }
        insts.push_back(std::move(I));
        dirty = true;
        if (out_handle) *out_handle = insts.back().handle;
        return GODAR_OK;
    }

    double skin_of(const Inst &I) const { return std::max(1.0, skin_frac * (I.rmax + I.prm.rtree)); }

    int attach_restore(int handle, std::shared_ptr<RestoreExtra> rx) {
        Inst *I = find(handle);
        if (!I || !I->pending) { set_err("restore needs a field not yet on the device"); return GODAR_ERR_STATE; }
        I->rx = std::move(rx);
        return GODAR_OK;
    }

    int remove(int handle) {
        for (size_t k = 0; k < insts.size(); k++)
            if (insts[k].handle == handle) {
                insts.erase(insts.begin() + k);
                dirty = true;
                return GODAR_OK;
            }
        set_err("unknown instance");
        return GODAR_ERR_NOT_FOUND;
    }

    // -------------------------------------------------------------- commit
    InstParams make_params(const Inst &I, long long coff, long long foff) const {
        const godar_params &p = I.prm;
        InstParams P{};
        P.dt = p.dt; P.rtree = p.rtree; P.skin = skin_of(I);
        P.rhoair = p.rhoair; P.rhoice = p.rhoice; P.rhowater = p.rhowater;
        P.Cdair = p.Cdair; P.Csair = p.Csair; P.Cdwater = p.Cdwater; P.Cswater = p.Cswater; P.z0w = p.z0w;
        P.ec = p.ec; P.gc = p.gc; P.beta = p.beta; P.pi = p.pi; P.sin_lat = p.sin_lat;
        P.mu = p.friction_coeff; P.sigmanc_crit = p.sigmanc_crit;
        P.eb = p.eb; P.lambda_rb = p.lambda_rb; P.lambda_lb = p.lambda_lb;
        P.sigmatb_crit = p.sigmatb_crit; P.sigmacb_crit = p.sigmacb_crit; P.tau_crit = p.tau_crit;
        P.dmax = p.dmax; P.dtd = p.dtd; P.dth = p.dth;
        P.ua = p.ua; P.va = p.va; P.uw = p.uw; P.vw = p.vw;
        P.nx = p.nx; P.ny = p.ny;
        P.log10z0 = dm::log(10.0 / p.z0w);
        P.log10z0f = logf(10.0f / (float)p.z0w);
        P.field_off = I.field.empty() ? -1 : foff;
        P.fnx = p.field_nx; P.fny = p.field_ny;
        P.slipping = p.slipping; P.ridging = p.ridging; P.shelter = p.shelter; P.cohesion = p.cohesion;
        P.boundary = p.boundary; P.bond_seed = p.bond_seed;
        P.n = I.n; P.off = I.off;
        const double R = I.rmax + p.rtree + P.skin;
        const double target = std::max(R / 2.0, 1e-6);
        P.ncx = std::max(1, std::min(4096, (int)std::floor(p.nx / target)));
        P.ncy = std::max(1, std::min(4096, (int)std::floor(p.ny / target)));
        P.cw = p.nx / P.ncx;
        P.ch = p.ny / P.ncy;
        P.kx = (int)std::ceil(R / P.cw);
        P.ky = (int)std::ceil(R / P.ch);
        P.coff = coff;
        P.f_dt = (float)p.dt;
        P.f_piec = (float)(p.pi * p.ec);
        P.f_ktc = (float)((6.0 * p.gc) / p.ec);
        P.f_beta = (float)p.beta;
        P.f_mu = (float)p.friction_coeff;
        P.f_sigc = (float)p.sigmanc_crit;
        P.f_llb = (float)p.lambda_lb;
        P.f_rhoipi = (float)(p.rhoice * p.pi);
        P.f_hfa = (float)((p.rhowater - p.rhoice) / p.rhowater);
        P.f_hfw = (float)(p.rhoice / p.rhowater);
        P.f_eb = (float)p.eb;
        P.f_inv_tau = (float)(1.0 / p.tau_crit);
        P.f_inv_sigcb = (float)(1.0 / p.sigmacb_crit);
        P.f_inv_sigtb = (float)(1.0 / p.sigmatb_crit);
        P.dt_dtd = p.dt / p.dtd;
        P.dt_dth = p.dt / p.dth;
        P.hfa_fac = (p.rhowater - p.rhoice) / p.rhowater;
        P.hfw_fac = p.rhoice / p.rhowater;
        return P;
    }

    int alloc_floe_set(FloeSet &f, int n) {
        auto ens = [&](Buf &b, size_t s) { return b.ensure(s, &bytes, &mp); };
        for (int s = 0; s < 2; s++) {
            Buf *dd[] = {&f.x[s], &f.y[s], &f.th[s], &f.u[s], &f.v[s], &f.om[s], &f.r[s], &f.h[s], &f.dtb1[s],
                         &f.dtb2[s], &f.thb1[s], &f.thb2[s], &f.x0[s], &f.y0[s]};
            for (Buf *b : dd) TRY(ens(*b, (size_t)n * 8));
            TRY(ens(f.id[s], (size_t)n * 4));
            TRY(ens(f.snap[s], (size_t)n * sizeof(Snap)));
        }
        return GODAR_OK;
    }

    int alloc_scratch(int n) {
        auto ens = [&](Buf &b, size_t s) { return b.ensure(s, &bytes, &mp); };
        TRY(ens(inst_b, (size_t)n * 4));
        TRY(ens(row_off2, (size_t)(n + 1) * 4)); TRY(ens(nlo2, (size_t)(n + 1) * 4));
        TRY(ens(up_off2, (size_t)(n + 1) * 4)); TRY(ens(lo_off2, (size_t)(n + 1) * 4));
        TRY(ens(nup, (size_t)(n + 1) * 4));
        TRY(ens(cnt, (size_t)(n + 1) * 4)); TRY(ens(old_slot, (size_t)n * 4));
        TRY(ens(keys, (size_t)n * 4)); TRY(ens(vals, (size_t)n * 4));
        TRY(ens(keys_alt, (size_t)n * 4)); TRY(ens(vals_alt, (size_t)n * 4));
        const size_t ntiles = (n + 2047) / 2048;
        TRY(ens(rs_counts, (256 * ntiles + 1) * 4));
        TRY(ens(scan_scratch, (256 * ntiles / 2048 + 64 + n / 2048 + 64) * 4));
        TRY(ens(diag, (size_t)14 * n * 8));
        TRY(ens(tmp_out, (size_t)n * 8));
        return GODAR_OK;
    }

    // Bond creation of the fresh fields with cohesion (bonds_init.cu) over
    // the admitted floes [s0, N), which sit on side 0 in reference order:
    // a cell list, each floe's bond count, their scan, and per field its
    // total (the field's nb).
    std::vector<BondRule> bond_rules(const std::vector<char> &fresh) const {
        std::vector<BondRule> r(insts.size());
        for (size_t k = 0; k < insts.size(); k++) {
            const godar_params &p = insts[k].prm;
            r[k].lim = p.bond_lim;
            r[k].lim_rel = p.bond_lim_rel;
            r[k].frac = p.bond_frac;
            r[k].seed = p.bond_seed;
            r[k].fresh = fresh[k] ? 1 : 0;
            r[k].boff = insts[k].boff;
            r[k].pad = 0;
        }
        return r;
    }

    int count_fresh_bonds(int s0, const std::vector<char> &fresh) {
        const int n = N - s0, ni = (int)insts.size();
        auto ens = [&](Buf &b, size_t sz) { return b.ensure(std::max<size_t>(sz, 16), &bytes, &mp); };
        TRY(ens(rule_b, (size_t)ni * sizeof(BondRule)));
        std::vector<BondRule> r = bond_rules(fresh);
        CK(cudaMemcpyAsync(rule_b.p, r.data(), r.size() * sizeof(BondRule), cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(cstart.p, 0, (size_t)C * 4, st));
        CK(cudaMemsetAsync(cend.p, 0, (size_t)C * 4, st));
        const int bits = std::max(1, ilog2ceil((uint64_t)std::max<long long>(C, 2)));
        launch_bond_init_count(views(), 0, s0, n, rule_b.as<BondRule>(), keys.as<uint32_t>(), vals.as<int>(),
                               keys_alt.as<uint32_t>(), vals_alt.as<int>(), bits, rs_counts.as<int>(),
                               scan_scratch.as<int>(), cstart.as<int>(), cend.as<int>(), cnt.as<int>(),
                               row_off2.as<int>(), st);
        // per fresh field: its bonds = scan[last] - scan[first]
        std::vector<int> fi, la, which;
        for (int k = 0; k < ni; k++)
            if (fresh[k]) {
                fi.push_back(insts[k].off - s0);
                la.push_back(insts[k].off + insts[k].n - s0);
                which.push_back(k);
            }
        const int m = (int)fi.size();
        TRY(ens(small_b, (size_t)3 * m * 4));
        int *d = small_b.as<int>();
        CK(cudaMemcpyAsync(d, fi.data(), (size_t)m * 4, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d + m, la.data(), (size_t)m * 4, cudaMemcpyHostToDevice, st));
        launch_bond_init_totals(row_off2.as<int>(), d, d + m, m, d + 2 * m, st);
        std::vector<int> tot(m);
        CK(cudaMemcpyAsync(tot.data(), d + 2 * m, (size_t)m * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        long long all = 0;
        for (int q = 0; q < m; q++) {
            if (tot[q] < 0) { set_err("bond count overflow"); return GODAR_ERR_CAPACITY; }
            insts[which[q]].nb = tot[q];
            all += tot[q];
        }
        if (all >= INT_MAX / 2) { set_err("too many bonds"); return GODAR_ERR_CAPACITY; }
        return GODAR_OK;
    }

    // Writes the fresh fields' bonds into the bond table (the cell list and
    // the scan of count_fresh_bonds are still in place).
    int fill_fresh_bonds(int s0, const std::vector<char> &fresh) {
        std::vector<BondRule> r = bond_rules(fresh);
        CK(cudaMemcpyAsync(rule_b.p, r.data(), r.size() * sizeof(BondRule), cudaMemcpyHostToDevice, st));
        launch_bond_init_fill(views(), 0, s0, N - s0, rule_b.as<BondRule>(), cstart.as<int>(), cend.as<int>(),
                              vals.as<int>(), row_off2.as<int>(), BS->bond_off.as<int>(), BS->bond_hi.as<int>(),
                              BS->bstat.as<BondStat>(), BS->bdyn[0].as<BondDyn>(), st);
        CK(cudaGetLastError());
        return GODAR_OK;
    }

    // Re-lays the batch after admissions/removals.  Resident instances move
    // device-to-device into fresh buffers (floes by the repack map, bonds by
    // the bond map); newly admitted ones are uploaded from their host copies;
    // the rebuild that follows carries contact histories over by reference
    // ids from the previous rows.
    int commit() {
        if (!dirty && have_rows) return GODAR_OK;
        // a relayout renumbers slots and sides: queued steps are read first
        // (a redo after an expiry among them may commit on its way)
        if (!pend.empty()) {
            TRY(resolve());
            if (!dirty && have_rows) return GODAR_OK;
        }
        cur_uvw.clear();
        TRY(wait_copy());
        TRY(sync_bonds());
        CK(cudaStreamSynchronize(st));
        const int oldN = N, oldNB = NB;
        const int ni = (int)insts.size();
        // bond tables of admitted fields: a restored field's own table, the
        // caller's restart list (geometry from the uploaded positions), or -
        // for a fresh field with cohesion - the bonds of time step 1, created
        // on the device once the floes are there (gpu_bonds)
        std::vector<HostBonds> bonds(ni);
        std::vector<char> gpu_bonds(ni, 0);
        std::vector<int> old_off(ni, -1), old_boff(ni, -1);
        int n_tot = 0, first_pending = -1;
        long long c_tot = 0, f_tot = 0;
        for (int k = 0; k < ni; k++) {
            Inst &I = insts[k];
            if (!I.pending) continue;
            if (I.rx) bonds[k] = I.rx->bonds;
            else if (I.fresh && I.prm.cohesion) gpu_bonds[k] = 1;
            else restart_bonds(I, bonds[k]);
        }
        for (int k = 0; k < ni; k++) {
            Inst &I = insts[k];
            if (I.pending) {
                I.nb = bonds[k].off.empty() ? 0 : bonds[k].off[I.n];
                if (first_pending < 0) first_pending = n_tot;
            } else {
                old_off[k] = I.off;
                old_boff[k] = I.boff;
            }
            I.off = n_tot;
            n_tot += I.n;
        }
        if ((long long)n_tot >= INT_MAX / 2) { set_err("too many floes"); return GODAR_ERR_CAPACITY; }
        std::vector<int> repack(n_tot, -1), hinst(n_tot);
        std::vector<InstParams> hp(ni);
        std::vector<double> hfield;
        for (int k = 0; k < ni; k++) {
            Inst &I = insts[k];
            for (int i = 0; i < I.n; i++) {
                hinst[I.off + i] = k;
                if (!I.pending) repack[I.off + i] = old_off[k] + i;
            }
            hp[k] = make_params(I, c_tot, f_tot);
            c_tot += (long long)hp[k].ncx * hp[k].ncy;
            if (!I.field.empty()) {
                hfield.insert(hfield.end(), I.field.begin(), I.field.end());
                f_tot += (long long)I.field.size();
            }
        }
        if (c_tot >= (1LL << 31)) { set_err("too many cells"); return GODAR_ERR_CAPACITY; }
        ridging_any = false;
        walls_any = false;
        for (const Inst &I : insts) {
            ridging_any = ridging_any || I.prm.ridging != 0;
            walls_any = walls_any || has_walls(I.prm.boundary);
        }
        const bool migrate = have_rows && oldN > 0;
        std::unique_ptr<FloeSet> oldF = std::move(F);
        std::unique_ptr<BondSet> oldB = std::move(BS);
        F = spareF ? std::move(spareF) : std::make_unique<FloeSet>();
        BS = spareB ? std::move(spareB) : std::make_unique<BondSet>();
        TRY(alloc_floe_set(*F, n_tot));
        TRY(alloc_scratch(n_tot));
        const int old_cur = cur;
        N = n_tot; C = c_tot;
        const int sn = 0;
        auto up = [&](void *dst, const void *src, size_t nbytes) -> int {
            if (nbytes) CK(cudaMemcpyAsync(dst, src, nbytes, cudaMemcpyHostToDevice, st));
            return GODAR_OK;
        };
        TRY(up(inst_b.p, hinst.data(), (size_t)N * 4));
        TRY(params_b.ensure(std::max<size_t>(hp.size(), 1) * sizeof(InstParams), &bytes, &mp));
        TRY(up(params_b.p, hp.data(), hp.size() * sizeof(InstParams)));
        hparams = hp;
        TRY(field_b.ensure(std::max<size_t>(hfield.size(), 1) * 8, &bytes, &mp));
        TRY(up(field_b.p, hfield.data(), hfield.size() * 8));
        TRY(cstart.ensure((size_t)std::max<long long>(C, 1) * 4, &bytes, &mp));
        TRY(cend.ensure((size_t)std::max<long long>(C, 1) * 4, &bytes, &mp));
        // resident floes, device to device
        TRY(repack_b.ensure((size_t)std::max(N, 1) * 4, &bytes, &mp));
        TRY(up(repack_b.p, repack.data(), (size_t)N * 4));
        Views Vn = views();
        if (oldF && oldN > 0) launch_gather_floes(make_views(*oldF, *oldB), old_cur, Vn, sn, repack_b.as<int>(), N, st);
        // admitted floes, host to device
        for (Inst &I : insts) {
            if (!I.pending) continue;
            const size_t o = (size_t)I.off, nb8 = (size_t)I.n * 8;
            TRY(up(F->x[sn].as<double>() + o, I.x.data(), nb8)); TRY(up(F->y[sn].as<double>() + o, I.y.data(), nb8));
            TRY(up(F->th[sn].as<double>() + o, I.th.data(), nb8)); TRY(up(F->u[sn].as<double>() + o, I.u.data(), nb8));
            TRY(up(F->v[sn].as<double>() + o, I.v.data(), nb8)); TRY(up(F->om[sn].as<double>() + o, I.om.data(), nb8));
            TRY(up(F->r[sn].as<double>() + o, I.r.data(), nb8)); TRY(up(F->h[sn].as<double>() + o, I.h.data(), nb8));
            if (I.rx) {
                TRY(up(F->dtb1[sn].as<double>() + o, I.rx->dtb1.data(), nb8));
                TRY(up(F->dtb2[sn].as<double>() + o, I.rx->dtb2.data(), nb8));
                TRY(up(F->thb1[sn].as<double>() + o, I.rx->thb1.data(), nb8));
                TRY(up(F->thb2[sn].as<double>() + o, I.rx->thb2.data(), nb8));
            } else {
                CK(cudaMemsetAsync(F->dtb1[sn].as<double>() + o, 0, nb8, st));
                CK(cudaMemsetAsync(F->dtb2[sn].as<double>() + o, 0, nb8, st));
                CK(cudaMemsetAsync(F->thb1[sn].as<double>() + o, 0, nb8, st));
                CK(cudaMemsetAsync(F->thb2[sn].as<double>() + o, 0, nb8, st));
            }
            std::vector<int> ids(I.n);
            std::iota(ids.begin(), ids.end(), 0);
            TRY(up(F->id[sn].as<int>() + o, ids.data(), (size_t)I.n * 4));
        }
        // bonds: the fresh fields' counts from the device, then every
        // field's place in the table (instances in layout order)
        if (std::any_of(gpu_bonds.begin(), gpu_bonds.end(), [](char c) { return c != 0; }))
            TRY(count_fresh_bonds(first_pending, gpu_bonds));
        int nb_tot = 0;
        for (Inst &I : insts) {
            I.boff = nb_tot;
            nb_tot += I.nb;
        }
        NB = nb_tot;
        std::vector<int> bmap(NB, -1);
        for (int k = 0; k < ni; k++)
            if (old_boff[k] >= 0)
                for (int q = 0; q < insts[k].nb; q++) bmap[insts[k].boff + q] = old_boff[k] + q;
        auto ens = [&](Buf &b, size_t sz) { return b.ensure(std::max<size_t>(sz, 16), &bytes, &mp); };
        TRY(ens(BS->bond_off, (size_t)(N + 1) * 4));
        TRY(ens(BS->bond_hi, (size_t)NB * 4));
        TRY(ens(BS->bstat, (size_t)NB * sizeof(BondStat)));
        TRY(ens(BS->bdyn[0], (size_t)NB * sizeof(BondDyn)));
        if (oldB && oldN > 0) {
            if (NB > 0 && oldNB > 0) {
                TRY(bmap_b.ensure((size_t)NB * 4, &bytes, &mp));
                TRY(up(bmap_b.p, bmap.data(), (size_t)NB * 4));
                launch_gather_bonds(oldB->bond_hi.as<int>(), oldB->bstat.as<BondStat>(),
                                    oldB->bdyn[0].as<BondDyn>(),
                                    BS->bond_hi.as<int>(), BS->bstat.as<BondStat>(), BS->bdyn[sn].as<BondDyn>(),
                                    bmap_b.as<int>(), NB, st);
            }
            std::vector<int> tab(4 * ni);
            for (int k = 0; k < ni; k++) {
                tab[k] = old_off[k];
                tab[ni + k] = insts[k].off;
                tab[2 * ni + k] = old_boff[k];
                tab[3 * ni + k] = insts[k].boff;
            }
            TRY(small_b.ensure((size_t)std::max(4 * ni, 4) * 4, &bytes, &mp));
            TRY(up(small_b.p, tab.data(), tab.size() * 4));
            const int *t4 = small_b.as<int>();
            launch_rebase_bond_off(oldB->bond_off.as<int>(), BS->bond_off.as<int>(), inst_b.as<int>(), t4, t4 + ni,
                                   t4 + 2 * ni, t4 + 3 * ni, N, st);
        }
        if (std::any_of(gpu_bonds.begin(), gpu_bonds.end(), [](char c) { return c != 0; }))
            TRY(fill_fresh_bonds(first_pending, gpu_bonds));
        for (int k = 0; k < ni; k++) {
            Inst &I = insts[k];
            if (!I.pending || gpu_bonds[k]) continue;
            const HostBonds &B = bonds[k];
            std::vector<int> off(I.n);
            for (int i = 0; i < I.n; i++) off[i] = I.boff + (B.off.empty() ? 0 : B.off[i]);
            TRY(up(BS->bond_off.as<int>() + I.off, off.data(), (size_t)I.n * 4));
            if (I.nb == 0) continue;
            std::vector<BondStat> hbs(I.nb);
            std::vector<BondDyn> hbd(I.nb);
            for (int q = 0; q < I.nb; q++) {
                BondDyn bd{};
                bd.dnb = B.dnb[q]; bd.dtb = B.dtb[q]; bd.thji = B.thji[q]; bd.thij = B.thij[q]; bd.dmg = B.dmg[q];
                bd.flag = B.flag[q];
                hbd[q] = bd;
                BondStat bs{};
                bs.rb = B.rb[q]; bs.hb = B.hb[q]; bs.lb = B.lb[q]; bs.sb = B.sb[q]; bs.ib = B.ib[q];
                const double EA = I.prm.eb * bs.sb, EI = I.prm.eb * bs.ib, L = bs.lb;
                bs.k_ax = (float)(EA / L);
                bs.k_sh1 = (float)((12.0 * EI) / ((L * L) * L));
                bs.k_sh2 = (float)((6.0 * EI) / (L * L));
                bs.k_r1 = (float)((4.0 * EI) / L);
                bs.k_r2 = (float)((2.0 * EI) / L);
                bs.ei_l = (float)(EI / L);
                bs.ea_l = (float)(EA * L);
                bs.inv_l = (float)(1.0 / L);
                hbs[q] = bs;
            }
            TRY(up(BS->bond_hi.as<int>() + I.boff, B.hi.data(), (size_t)I.nb * 4));
            TRY(up(BS->bstat.as<BondStat>() + I.boff, hbs.data(), (size_t)I.nb * sizeof(BondStat)));
            TRY(up(BS->bdyn[sn].as<BondDyn>() + I.boff, hbd.data(), (size_t)I.nb * sizeof(BondDyn)));
        }
        TRY(up(BS->bond_off.as<int>() + N, &NB, sizeof(int)));
        CK(cudaStreamSynchronize(st));
        for (auto &I : insts) {
            if (I.pending) {
                I.pending = false;
                std::vector<double>().swap(I.x); std::vector<double>().swap(I.y);
                std::vector<double>().swap(I.r); std::vector<double>().swap(I.h);
                std::vector<double>().swap(I.th); std::vector<double>().swap(I.om);
                std::vector<double>().swap(I.u); std::vector<double>().swap(I.v);
                std::vector<int>().swap(I.bi); std::vector<int>().swap(I.bj);
                std::vector<double>().swap(I.dmg);
            }
        }
        dirty = false;
        cur = sn;
        TRY(rebuild(migrate ? repack_b.as<int>() : nullptr, migrate ? oldF->id[old_cur].as<int>() : nullptr,
                    migrate));
        TRY(inject_restored_histories());
        CK(cudaStreamSynchronize(st));
        if (oldF) spareF = std::move(oldF);
        if (oldB) spareB = std::move(oldB);
        return GODAR_OK;
    }

    // Pair histories of instances restored from a checkpoint, into the rows
    // just built; the mixed path's contact list is built again so that it
    // knows which pairs carry a history.
    int inject_restored_histories() {
        bool any = false;
        for (Inst &I : insts) {
            if (!I.rx) continue;
            const int nh = (int)I.rx->hi.size();
            if (nh > 0) {
                Buf pi, pj, h4, so;
                TRY(pi.ensure((size_t)nh * 4, nullptr)); TRY(pj.ensure((size_t)nh * 4, nullptr));
                TRY(h4.ensure((size_t)nh * 32, nullptr)); TRY(so.ensure((size_t)std::max(N, 1) * 4, nullptr));
                CK(cudaMemcpyAsync(pi.p, I.rx->hi.data(), (size_t)nh * 4, cudaMemcpyHostToDevice, st));
                CK(cudaMemcpyAsync(pj.p, I.rx->hj.data(), (size_t)nh * 4, cudaMemcpyHostToDevice, st));
                CK(cudaMemcpyAsync(h4.p, I.rx->h4.data(), (size_t)nh * 32, cudaMemcpyHostToDevice, st));
                const bool fp64 = prec == GODAR_PREC_FP64;
                launch_hist_inject(views(), cur, I.off, nh, pi.as<int>(), pj.as<int>(), h4.as<double>(), so.as<int>(),
                                   fp64 ? 1 : 0, 0, fp64 ? nullptr : pfl.as<unsigned char>(), st);
                CK(cudaStreamSynchronize(st));
                any = true;
            }
            I.rx.reset();
        }
        if (any && prec != GODAR_PREC_FP64) TRY(contact_list(cur, (int)E));
        if (any && prec == GODAR_PREC_FP64) TRY(fp64_rows(cur));
        return GODAR_OK;
    }

    // Everything a field needs to continue exactly: floe state and wall
    // histories in reference order, the bond table, the pair histories.
    int checkpoint(int handle, std::vector<char> &out) {
        Inst *I = find(handle);
        if (!I) { set_err("unknown instance"); return GODAR_ERR_NOT_FOUND; }
        if (I->pending) TRY(commit());
        TRY(wait_copy());
        TRY(sync_bonds());
        const int n = I->n;
        const bool fp64 = prec == GODAR_PREC_FP64;
        Views V = views();
        // floe state: x y u v r h theta omega, then the wall histories
        std::vector<double> st12((size_t)12 * n);
        const int codes[12] = {0, 1, 2, 3, 4, 5, 6, 7, GATHER_DTB1, GATHER_DTB1 + 1, GATHER_DTB1 + 2, GATHER_DTB1 + 3};
        for (int f = 0; f < 12; f++) {
            launch_gather_field(V, cur, 0, I->off, n, codes[f], tmp_out.as<double>(), st);
            CK(cudaMemcpyAsync(st12.data() + (size_t)f * n, tmp_out.p, (size_t)n * 8, cudaMemcpyDeviceToHost, st));
        }
        // bond table of the instance (CSR over its reference ids)
        const int nb = I->nb;
        std::vector<int> boff(n + 1), bhi(nb);
        std::vector<BondStat> bst(nb);
        std::vector<BondDyn> bdy(nb);
        CK(cudaMemcpyAsync(boff.data(), BS->bond_off.as<int>() + I->off, (size_t)(n + 1) * 4, cudaMemcpyDeviceToHost, st));
        if (nb) {
            CK(cudaMemcpyAsync(bhi.data(), BS->bond_hi.as<int>() + I->boff, (size_t)nb * 4, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(bst.data(), BS->bstat.as<BondStat>() + I->boff, (size_t)nb * sizeof(BondStat),
                               cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(bdy.data(), BS->bdyn[0].as<BondDyn>() + I->boff, (size_t)nb * sizeof(BondDyn),
                               cudaMemcpyDeviceToHost, st));
        }
        // pair histories: count, then fill
        CK(cudaMemsetAsync(tmp_cnt.p, 0, sizeof(int), st));
        launch_hist_list(V, cur, I->off, n, fp64 ? 1 : 0, 0, tmp_cnt.as<int>(), nullptr, nullptr,
                         nullptr, 0, st);
        int nh = 0;
        CK(cudaMemcpyAsync(&nh, tmp_cnt.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        std::vector<int> hi(nh), hj(nh);
        std::vector<double> h4((size_t)4 * nh);
        if (nh) {
            Buf pi, pj, hb;
            TRY(pi.ensure((size_t)nh * 4, nullptr)); TRY(pj.ensure((size_t)nh * 4, nullptr));
            TRY(hb.ensure((size_t)nh * 32, nullptr));
            CK(cudaMemsetAsync(tmp_cnt.p, 0, sizeof(int), st));
            launch_hist_list(V, cur, I->off, n, fp64 ? 1 : 0, 0, tmp_cnt.as<int>(), pi.as<int>(),
                             pj.as<int>(), hb.as<double>(), nh, st);
            CK(cudaMemcpyAsync(hi.data(), pi.p, (size_t)nh * 4, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(hj.data(), pj.p, (size_t)nh * 4, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(h4.data(), hb.p, (size_t)nh * 32, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            // a fixed order, whatever order the kernel found them in
            std::vector<int> ord(nh);
            std::iota(ord.begin(), ord.end(), 0);
            std::sort(ord.begin(), ord.end(), [&](int a, int b) {
                return hi[a] != hi[b] ? hi[a] < hi[b] : hj[a] < hj[b];
            });
            std::vector<int> hi2(nh), hj2(nh);
            std::vector<double> h42((size_t)4 * nh);
            for (int k = 0; k < nh; k++) {
                hi2[k] = hi[ord[k]]; hj2[k] = hj[ord[k]];
                for (int c = 0; c < 4; c++) h42[4 * (size_t)k + c] = h4[4 * (size_t)ord[k] + c];
            }
            hi.swap(hi2); hj.swap(hj2); h4.swap(h42);
        }
        // layout: header, floe arrays, bonds (i j flag pad, then 10 doubles), histories (i j, then 4 doubles)
        CkptHeader hd{};
        std::memcpy(hd.magic, "GODARCK1", 8);
        hd.version = 1; hd.precision = prec; hd.n = n; hd.nb = nb; hd.nh = nh;
        out.clear();
        auto put = [&](const void *p, size_t b) { const char *c = (const char *)p; out.insert(out.end(), c, c + b); };
        put(&hd, sizeof(hd));
        put(st12.data(), st12.size() * 8);
        for (int i = 0; i < n; i++)
            for (int b = boff[i] - I->boff; b < boff[i + 1] - I->boff; b++) {
                const int32_t ij[4] = {i, bhi[b], bdy[b].flag, 0};
                const double v[10] = {bst[b].rb, bst[b].hb, bst[b].lb, bst[b].sb, bst[b].ib,
                                      bdy[b].dnb, bdy[b].dtb, bdy[b].thji, bdy[b].thij, bdy[b].dmg};
                put(ij, sizeof(ij));
                put(v, sizeof(v));
            }
        for (int k = 0; k < nh; k++) {
            const int32_t ij[2] = {hi[k], hj[k]};
            put(ij, sizeof(ij));
            put(&h4[4 * (size_t)k], 32);
        }
        return GODAR_OK;
    }

    // -------------------------------------------------------------- kernel (a)
    // Rebuilds the neighbour rows from the state on side cur; the new cell
    // order lands on side cur ^ 1, which becomes current.  repack/old_ids
    // describe the previous layout when the batch was re-laid (commit).
    // Host wall time of every rebuild, to its end on the device.
    int rebuild(const int *repack, const int *old_ids, bool migrate_from_old) {
        const auto t0 = std::chrono::steady_clock::now();
        int rc = rebuild_rows(repack, old_ids, migrate_from_old);
        if (rc == GODAR_OK && cudaStreamSynchronize(st) != cudaSuccess) { cudaGetLastError(); rc = GODAR_ERR_CUDA; }
        rebuild_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return rc;
    }

    int rebuild_rows(const int *repack, const int *old_ids, bool migrate_from_old) {
        if (N == 0) { have_rows = true; return GODAR_OK; }
        TRY(sync_bonds());
        Views V = views();
        const int nxt = cur ^ 1;
        const bool have_old = have_rows && (repack ? migrate_from_old : true);
        launch_cell_keys(V, cur, keys.as<uint32_t>(), vals.as<int>(), st);
        const int bits = std::max(1, ilog2ceil((uint64_t)std::max<long long>(C, 2)));
        radix_sort(keys.as<uint32_t>(), vals.as<int>(), keys_alt.as<uint32_t>(), vals_alt.as<int>(), N, bits,
                   rs_counts.as<int>(), scan_scratch.as<int>(), st);
        launch_permute(V, cur, vals.as<int>(), repack, old_slot.as<int>(), st);
        CK(cudaMemsetAsync(cstart.p, 0, (size_t)C * 4, st));
        CK(cudaMemsetAsync(cend.p, 0, (size_t)C * 4, st));
        launch_cell_ranges(keys.as<uint32_t>(), N, cstart.as<int>(), cend.as<int>(), st);
        launch_nbr_count(V, nxt, cstart.as<int>(), cend.as<int>(), cnt.as<int>(), st);
        scan_excl(cnt.as<int>(), row_off2.as<int>(), N, scan_scratch.as<int>(), st);
        int Enew = 0;
        CK(cudaMemcpyAsync(&Enew, row_off2.as<int>() + N, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (Enew < 0) { set_err("neighbour rows overflow int32"); return GODAR_ERR_CAPACITY; }
        if (Enew % 2) { set_err("asymmetric neighbour rows"); return GODAR_ERR_CAPACITY; }
        const int Pn = Enew / 2;
        const size_t he = hist_elem();
        auto ens = [&](Buf &b, size_t s) { return b.ensure(std::max<size_t>(s, 16), &bytes, &mp); };
        TRY(ens(ent2, (size_t)Enew * 8)); TRY(ens(dist2, (size_t)Enew * 8));
        TRY(ens(ent_up2, (size_t)Pn * 8)); TRY(ens(ent_lo2, (size_t)Pn * 8));
        TRY(ens(bidx2, (size_t)Pn * 4)); TRY(ens(hist2, (size_t)Pn * he));
        launch_nbr_fill(V, nxt, cstart.as<int>(), cend.as<int>(), row_off2.as<int>(), ent2.as<int2>(),
                        dist2.as<double>(), nlo2.as<int>(), prec == GODAR_PREC_FP64 ? 0 : 1, st);
        launch_nbr_link(V, row_off2.as<int>(), nlo2.as<int>(), ent2.as<int2>(), st);
        // split into owner and partner rows
        launch_row_lengths(N, row_off2.as<int>(), nlo2.as<int>(), nup.as<int>(), st);
        scan_excl(nlo2.as<int>(), lo_off2.as<int>(), N, scan_scratch.as<int>(), st);
        scan_excl(nup.as<int>(), up_off2.as<int>(), N, scan_scratch.as<int>(), st);
        launch_split_rows(N, row_off2.as<int>(), nlo2.as<int>(), ent2.as<int2>(), lo_off2.as<int>(), up_off2.as<int>(), ent_lo2.as<int2>(), ent_up2.as<int2>(), st);
        const bool fp64 = prec == GODAR_PREC_FP64;
        {
            // without a previous generation of rows every history starts at zero
            const int *o_up_off = have_old ? up_off.as<int>() : nullptr;
            const int *o_id = old_ids ? old_ids : F->id[cur].as<int>();
            launch_migrate(V, fp64, nxt, old_slot.as<int>(), o_up_off, ent_up.as<int2>(), o_id,
                           hist[0].p, up_off2.as<int>(), ent_up2.as<int2>(), hist2.p, bidx2.as<int>(), st);
            CK(cudaStreamSynchronize(st));
        }
        // the new generation becomes the primary rows
        if ((long long)Pn > Ecap) {
            CK(cudaStreamSynchronize(st));
            const long long cap = (long long)(Pn * 1.25) + 1024;
            Buf *pb[] = {&ent_up, &ent_lo, &bidx, &hist[0], &edist, &pdn, &erow_up, &lo_of, &pfl, &lfl,
                         &prec_b, &prx_b, &pdg_b, &work_b, &work_st_b, &clist_b, &cscan_b, &frec_b, &fwork1_b,
                         &flisted_b, &fpart_b, &fplist_b};
            for (Buf *b : pb) b->release(&bytes);
            TRY(ens(ent_up, cap * 8)); TRY(ens(ent_lo, cap * 8)); TRY(ens(bidx, cap * 4));
            TRY(ens(hist[0], cap * he)); TRY(ens(pdn, cap * 4));
            if (fp64) {
                TRY(ens(edist, cap * 8));
                TRY(ens(erow_up, cap * 4)); TRY(ens(pfl, cap + 16));
                TRY(ens(work_b, cap * sizeof(FP64Item))); TRY(ens(fwork1_b, cap * sizeof(FP64Item)));
                TRY(ens(frec_b, cap * FP64_PAIR_REC_BYTES));
                TRY(ens(flisted_b, cap + 16)); TRY(ens(fpart_b, cap * 16)); TRY(ens(fplist_b, cap * 4));
            } else {
                TRY(ens(erow_up, cap * 4)); TRY(ens(lo_of, cap * 4));
                // flag bytes are read in aligned 8-byte words
                TRY(ens(pfl, cap + 16)); TRY(ens(lfl, cap + 16)); TRY(ens(work_b, cap * 4)); TRY(ens(work_st_b, cap * 8));
                // the contact list: {entry, bound} for every item, then {slots}
                TRY(ens(clist_b, cap * 16)); TRY(ens(cscan_b, (cap / 2048 + 16) * 4));
                TRY(ens(prec_b, cap * 32)); TRY(ens(prx_b, cap * 8)); TRY(ens(pdg_b, cap * 32));
            }
            Ecap = cap;
        }
        if (up_off.bytes < (size_t)(N + 1) * 4 || lo_off.bytes < (size_t)(N + 1) * 4) {
            CK(cudaStreamSynchronize(st));
            TRY(ens(up_off, (size_t)(N + 1) * 4));
            TRY(ens(lo_off, (size_t)(N + 1) * 4));
        }
        CK(cudaMemcpyAsync(up_off.p, up_off2.p, (size_t)(N + 1) * 4, cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(lo_off.p, lo_off2.p, (size_t)(N + 1) * 4, cudaMemcpyDeviceToDevice, st));
        if (Pn) {
            CK(cudaMemcpyAsync(ent_up.p, ent_up2.p, (size_t)Pn * 8, cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(ent_lo.p, ent_lo2.p, (size_t)Pn * 8, cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(bidx.p, bidx2.p, (size_t)Pn * 4, cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(hist[0].p, hist2.p, (size_t)Pn * he, cudaMemcpyDeviceToDevice, st));
            CK(cudaMemsetAsync(pdn.p, 0xff, (size_t)Pn * 4, st));
        }
        launch_copy_ids(V, nxt, st);
        launch_fill_erow(up_off.as<int>(), N, erow_up.as<unsigned>(), st);
        if (fp64) {
            E = Pn;
            TRY(fp64_rows(nxt));
        }
        TRY(nwork_b.ensure(16, &bytes, &mp));
        CK(cudaMemsetAsync(nwork_b.p, 0, 2 * sizeof(int), st));
        // per-floe sums: the FP64 path's ordered record sums, the mixed path's window partials
        TRY(fsum_b.ensure((size_t)N * (fp64 ? 8 * FP64_FLOE_SUMS : 32), &bytes, &mp));
        if (!fp64) {
            launch_mixed_rows_init(Pn, ent_lo.as<int2>(), hist[0].p, lo_of.as<int>(), pfl.as<unsigned char>(),
                                   lfl.as<unsigned char>(), st);
            TRY(frex_b.ensure((size_t)N * 4, &bytes, &mp));
            TRY(fdg_b.ensure((size_t)N * 32, &bytes, &mp));
            launch_pack_snap(V, nxt, st);
            TRY(contact_list(nxt, Pn));
            TRY(mixed_bond_lists(nxt));
            // the contact list holds the gaps at the rebuild: D starts at zero
            CK(cudaMemsetAsync(dsp_b.p, 0, 4 * sizeof(unsigned), st));
        }
        E = Pn;
        cur = nxt;
        rebuilds++;
        gbase = 0;
        TRY(reset_status());
        have_rows = true;
        CK(cudaGetLastError());
        return GODAR_OK;
    }

    // Mixed path: the contact list of the rows just built (P owner entries,
    // floes on side `side`); the second-generation rows are free scratch by
    // then (marks and positions).
    int contact_list(int side, int P) {
        Ec = 0;
        if (P <= 0) return GODAR_OK;
        int *mark = ent2.as<int>(), *pos = mark + P;
        launch_contact_list(views(), side, P, erow_up.as<unsigned>(), pfl.as<unsigned char>(), mark, pos,
                            cscan_b.as<int>(), clist_b.as<int2>(), clist_b.as<int2>() + Ecap, st);
        int ec = 0;
        CK(cudaMemcpyAsync(&ec, pos + P, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        Ec = ec;
        return GODAR_OK;
    }

    // FP64 path, after every rebuild (E owner entries, floes on side `side`)
    // and after a restore injects histories: the pairs a plain step must
    // visit, at the head of every row, and the screen's list of them.
    int fp64_rows(int side) {
        auto ens = [&](Buf &b, size_t sz) { return b.ensure(std::max<size_t>(sz, 16), &bytes, &mp); };
        TRY(ens(fupn_b, (size_t)N * 4)); TRY(ens(flon_b, (size_t)N * 4)); TRY(ens(fpos_b, (size_t)(N + 1) * 4));
        launch_fp64_rows(views(), side, (int)E, erow_up.as<unsigned>(), flisted_b.as<unsigned char>(),
                         fupn_b.as<int>(), flon_b.as<int>(), fpart_b.as<int2>(), fpos_b.as<int>(),
                         scan_scratch.as<int>(), fplist_b.as<int>(), st);
        int lc = 0;
        CK(cudaMemcpyAsync(&lc, fpos_b.as<int>() + N, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        CK(cudaGetLastError());
        Lc = lc;
        return GODAR_OK;
    }

    // -------------------------------------------------------------- stepping
    MixedBufs mixed_bufs() {
        MixedBufs B;
        B.pfl = pfl.as<unsigned char>(); B.lfl = lfl.as<unsigned char>(); B.lo_of = lo_of.as<int>();
        B.rec = prec_b.as<float4>(); B.rx = prx_b.as<float2>(); B.pdg = pdg_b.as<float4>();
        B.brec = brec.as<float4>(); B.bdg = bdg.as<float4>(); B.bsp = wsp_b.as<int4>(); B.wdyn = wdyn_b.as<BondDyn>(); B.winv = winv_b.as<int>();
        B.blo_start = blo_start.as<int>(); B.blo_end = blo_end.as<int>(); B.blo_idx = bvals.as<int>();
        B.work = work_b.as<int>(); B.nwork = nwork_b.as<int>(); B.work_st = work_st_b.as<int2>();
        B.bfo = bfo.as<int>(); B.bst = bst32.as<BondGeom32>();
        B.fsum = fsum_b.as<float4>(); B.frex = frex_b.as<float>(); B.fdg = fdg_b.as<float4>();
        B.dsp = dsp_b.as<unsigned>();
        return B;
    }

    // Mixed path, after every rebuild: the slots of both floes of every bond
    // and, per floe, the bonds in which it is the higher id (a stable sort of
    // the bonds by the partner's global id); bond records start at zero.
    // Writes the bond kernel's working records back to the bond table.
    int sync_bonds() {
        if (prec != GODAR_PREC_FP64 && wdirty && wnb > 0 && BS)
            launch_bond_work_scatter(perm_b.as<int>(), wnb, wdyn_b.as<BondDyn>(), BS->bdyn[0].as<BondDyn>(), st);
        wdirty = false;
        CK(cudaGetLastError());
        return GODAR_OK;
    }

    int mixed_bond_lists(int side) {
        auto ens = [&](Buf &b, size_t sz) { return b.ensure(std::max<size_t>(sz, 16), &bytes, &mp); };
        TRY(ens(slot_of, (size_t)N * 4)); TRY(ens(blo_start, (size_t)N * 4)); TRY(ens(blo_end, (size_t)N * 4));
        TRY(ens(bfo, (size_t)(N + 1) * 4));
        CK(cudaMemsetAsync(blo_start.p, 0, (size_t)N * 4, st));
        CK(cudaMemsetAsync(blo_end.p, 0, (size_t)N * 4, st));
        if (NB == 0) {
            CK(cudaMemsetAsync(bfo.p, 0, (size_t)(N + 1) * 4, st));
            return GODAR_OK;
        }
        const size_t nt = ((size_t)NB + 2047) / 2048;
        TRY(ens(brec, (size_t)NB * 32)); TRY(ens(bdg, (size_t)NB * 64)); TRY(ens(bsp, (size_t)NB * 16));
        TRY(ens(bst32, (size_t)NB * sizeof(BondGeom32)));
        TRY(ens(bflag_b, (size_t)NB * 2));
        TRY(ens(wdyn_b, (size_t)NB * sizeof(BondDyn))); TRY(ens(wsp_b, (size_t)NB * 16));
        TRY(ens(winv_b, (size_t)NB * 4)); TRY(ens(perm_b, (size_t)NB * 4)); TRY(ens(wfo_b, (size_t)(N + 1) * 4));
        TRY(ens(bkeys, (size_t)NB * 4)); TRY(ens(bvals, (size_t)NB * 4));
        TRY(ens(bkeys_alt, (size_t)NB * 4)); TRY(ens(bvals_alt, (size_t)NB * 4));
        TRY(ens(brs_counts, (256 * nt + 1) * 4));
        TRY(ens(bscan, (256 * nt / 2048 + 64 + (size_t)NB / 2048 + 64) * 4));
        Views V = views();
        launch_bond_slots(V, side, slot_of.as<int>(), bsp.as<int4>(), bkeys.as<uint32_t>(), bvals.as<int>(), st);
        const int bits = std::max(1, ilog2ceil((uint64_t)std::max(N, 2)));
        radix_sort(bkeys.as<uint32_t>(), bvals.as<int>(), bkeys_alt.as<uint32_t>(), bvals_alt.as<int>(), NB, bits,
                   brs_counts.as<int>(), bscan.as<int>(), st);
        launch_cell_ranges(bkeys.as<uint32_t>(), NB, blo_start.as<int>(), blo_end.as<int>(), st);
        launch_bond_positions(V, side, blo_start.as<int>(), blo_end.as<int>(), bvals.as<int>(), cnt.as<int>(),
                              bfo.as<int>(), scan_scratch.as<int>(), bsp.as<int4>(), st);
        CK(cudaMemsetAsync(brec.p, 0, (size_t)NB * 32, st));
        launch_bond_work(V, side, NB, cnt.as<int>(), wfo_b.as<int>(), scan_scratch.as<int>(), perm_b.as<int>(),
                         BS->bstat.as<BondStat>(), BS->bdyn[0].as<BondDyn>(), bsp.as<int4>(), bst32.as<BondGeom32>(),
                         wdyn_b.as<BondDyn>(), wsp_b.as<int4>(), winv_b.as<int>(), bflag_b.as<unsigned char>(), st);
        wnb = NB;
        wdirty = false;
        return GODAR_OK;
    }

    void drop_graphs() {
        for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
        graphs.clear();
        graph_uses.clear();
    }

    // Event record that also works inside a stream capture (as a graph node).
    int record(cudaEvent_t e, bool capturing, cudaStream_t s = nullptr) {
        if (!s) s = st;
        if (capturing) CK(cudaEventRecordWithFlags(e, s, cudaEventRecordExternal));
        else CK(cudaEventRecord(e, s));
        return GODAR_OK;
    }

    bool concurrent_bonds() const { return overlap_bonds && prec != GODAR_PREC_FP64 && NB > 0 && E > 0 && !ridging_any; }

    // One time step with block sizes bs[]; ev (NEV events, optional)
    // brackets its kernels: [start, screen done, work list done, bonds
    // joined, sums done, step done, bonds done (second stream)].
    int launch_one(int side, int diag, int sic, const int *bs, cudaEvent_t *ev, bool capturing) {
        Views V = views();
        // a batch whose floe kernels fill at most half the GPU's threads has
        // short kernels, and the gap between two of them is a large part of
        // its step: each step kernel is scheduled while the one before it
        // finishes (programmatic dependent launch).  On larger batches that
        // made the step slower (0.362 against 0.354 ms on 2.2 M floes).
        V.pdl = step_pdl() && N <= PDL_MAX_FLOES;
        if (ev) TRY(record(ev[0], capturing));
        if (prec == GODAR_PREC_FP64) {
            FP64Lists L;
            L.work[0] = work_b.as<FP64Item>();
            L.work[1] = fwork1_b.as<FP64Item>();
            L.n = nwork_b.as<int>();
            // a plain step visits the pairs that can act before the next
            // rebuild; a diagnostic step every owner entry
            launch_pairs_fp64_screen(V, side, diag, diag ? (int)E : (int)Lc, diag ? nullptr : fplist_b.as<int>(),
                                     erow_up.as<unsigned>(), pfl.as<unsigned char>(), L, frec_b.p, cfg_block(bs[0]),
                                     cfg_variant(bs[0]), st);
            if (ev) TRY(record(ev[1], capturing));
            for (int l = 0; l < 2; l++) {
                launch_pairs_fp64_work(V, side, diag, l, (int)E, pfl.as<unsigned char>(), L, frec_b.p,
                                       cfg_block(bs[1 + l]), st);
                if (ev) TRY(record(ev[2 + l], capturing));
            }
            launch_row_sums_fp64(V, side, diag, pfl.as<unsigned char>(), frec_b.p, flon_b.as<int>(),
                                 fupn_b.as<int>(), fsum_b.as<double>(), cfg_block(bs[3]), st);
            if (ev) TRY(record(ev[4], capturing));
            launch_floes_fp64(V, side, diag, sic, fsum_b.as<double>(), nwork_b.as<int>(), cfg_block(bs[4]), st);
            if (ev)
                for (int q = 5; q < NEV; q++) TRY(record(ev[q], capturing));
        } else {
            MixedBufs B = mixed_bufs();
            // live-bond flags ping-pong with the floe state's side
            if (NB > 0) wdirty = true;
            B.bfl_rd = bflag_b.as<unsigned char>() + (size_t)side * NB;
            B.bfl_wr = bflag_b.as<unsigned char>() + (size_t)(side ^ 1) * NB;
            const bool conc = concurrent_bonds();
            if (conc) {
                CK(cudaEventRecord(ev_fork, st));
                CK(cudaStreamWaitEvent(st2, ev_fork, 0));
                launch_bonds_mixed(V, side, diag, NB, B, cfg_block(bs[2]), cfg_variant(bs[2]), test_wait_spins, st2);
                if (ev) TRY(record(ev[6], capturing, st2));
                CK(cudaEventRecord(ev_join, st2));
            }
            // the screen walks the contact list, or every entry on a diagnostic step
            launch_pairs_screen(V, side, diag, diag ? (int)E : (int)Ec, diag ? nullptr : clist_b.as<int2>(),
                                clist_b.as<int2>() + Ecap, B, cfg_block(bs[0]), cfg_variant(bs[0]), st);
            if (ev) TRY(record(ev[1], capturing));
            launch_pairs_work(V, side, diag, (int)E, erow_up.as<unsigned>(), B, cfg_block(bs[1]), st);
            if (ev) TRY(record(ev[2], capturing));
            if (conc) CK(cudaStreamWaitEvent(st, ev_join, 0));
            else launch_bonds_mixed(V, side, diag, NB, B, cfg_block(bs[2]), cfg_variant(bs[2]), test_wait_spins, st);
            if (ev) TRY(record(ev[3], capturing));
            launch_floe_sums(V, diag, B, cfg_block(bs[3]), st);
            if (ev) TRY(record(ev[4], capturing));
            launch_floes_mixed(V, side, diag, sic, walls_any ? 1 : 0, B, cfg_block(bs[4]), st);
            if (ev) TRY(record(ev[5], capturing));
        }
        return GODAR_OK;
    }

    int max_cfg() const {
        int m = 1;
        for (int q = 0; q < NPH; q++) m = std::max(m, ncfg[q]);
        return m;
    }

    int kernels_per_step() const {
        return prec == GODAR_PREC_FP64 ? 5 : (E > 0 ? 2 : 0) + (NB > 0 ? 1 : 0) + 2;
    }

    // The graph of K steps from side c0, captured on first use.  Returns
    // null (and turns graphs off) where capture is not available.
    cudaGraphExec_t capture(int K, int c0, int diag_last, const int *bs, int every) {
        while ((int)kev.size() < NEV * K) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) { cudaGetLastError(); return nullptr; }
            kev.push_back(e);
        }
        if (graph_gen != rebuilds) {
            drop_graphs();
            graph_gen = rebuilds;
        }
        const auto key = std::make_tuple(K, c0, diag_last | (every << 1));
        auto it = graphs.find(key);
        if (it != graphs.end()) return it->second;
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ex = nullptr;
        bool ok = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            int rc = GODAR_OK;
            for (int k = 0; k < K && rc == GODAR_OK; k++)
                rc = launch_one(c0 ^ (k & 1), (diag_last && k == K - 1) ? 1 : 0, k, bs,
                                (every > 0 && k % every == 0) ? &kev[NEV * k] : nullptr, true);
            ok = cudaStreamEndCapture(st, &g) == cudaSuccess && rc == GODAR_OK && g;
        }
        if (ok) ok = cudaGraphInstantiate(&ex, g, 0) == cudaSuccess;
        if (g) cudaGraphDestroy(g);
        if (!ok) {
            // capture is not available here: launch directly from now on
            cudaGetLastError();
            graphs_on = false;
            if (ex) cudaGraphExecDestroy(ex);
            return nullptr;
        }
        graphs.emplace(key, ex);
        return ex;
    }

    // Captures ahead of time the graphs that run(nsteps) will use if no
    // neighbour list expires on the way (the chunk schedule is known).
    int reserve(size_t want) {
        if (!mp.pool || want == 0) return GODAR_OK;
        size_t held = 0;
        CK(cudaMemPoolGetAttribute(mp.pool, cudaMemPoolAttrReservedMemCurrent, &held));
        if (held >= want) return GODAR_OK;
        void *p = nullptr;
        cudaError_t e = cudaMallocFromPoolAsync(&p, want - held, mp.pool, st);
        if (e != cudaSuccess) { cudaGetLastError(); g_last_error = std::string("reserve: ") + cudaGetErrorString(e); return GODAR_ERR_NOMEM; }
        CK(cudaFreeAsync(p, st));
        CK(cudaStreamSynchronize(st));
        return GODAR_OK;
    }

    int prepare(int nsteps) {
        TRY(commit());
        if (N == 0 || nsteps <= 0 || !graphs_on || tune_left > 0) return GODAR_OK;
        int c = cur, remaining = nsteps, ch = chunk;
        while (remaining > 0 && graphs_on) {
            int K = std::min(remaining, ch);
            while (K & (K - 1)) K &= K - 1;
            capture(K, c, (diagnostics && remaining == K) ? 1 : 0, blk, phase_every);
            c ^= (K & 1);
            remaining -= K;
            ch = std::min(ch * 2, 256);
        }
        return GODAR_OK;
    }

    // Launches K steps from side c0 (diagnostics on the last one if
    // diag_last) directly or through a captured graph.
    // every > 0: steps k of the chunk with k % every == 0 record the timing
    // events kev[NEV k ...].
    int launch_chunk(int K, int c0, int diag_last, const int *bs, bool tuning, int every) {
        while ((int)kev.size() < NEV * K) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            kev.push_back(e);
        }
        const bool pow2 = (K & (K - 1)) == 0;
        if (graphs_on && !tuning && pow2) {
            if (graph_gen != rebuilds) {
                drop_graphs();
                graph_gen = rebuilds;
            }
            // a chunk shape is captured the second time it runs in one
            // generation of rows (a batch whose membership changes every few
            // chunks would otherwise pay for captures it never reuses)
            const auto key = std::make_tuple(K, c0, diag_last | (every << 1));
            const bool have = graphs.count(key) != 0;
            cudaGraphExec_t ex = (have || graph_uses[key]++ >= 1) ? capture(K, c0, diag_last, bs, every) : nullptr;
            if (ex) {
                CK(cudaGraphLaunch(ex, st));
                graph_launches++;
                return GODAR_OK;
            }
        }
        for (int k = 0; k < K; k++)
            TRY(launch_one(c0 ^ (k & 1), (diag_last && k == K - 1) ? 1 : 0, k, bs,
                           (every > 0 && k % every == 0) ? &kev[NEV * k] : nullptr, false));
        return GODAR_OK;
    }

    // Advances every instance by nsteps; diagnostics on the last step.
    int run(int nsteps) {
        TRY(commit());
        if (N == 0 || nsteps <= 0) return GODAR_OK;
        // a step writes the other side: it waits for the gathers that read
        // that side (one step from the gathered side only reads it)
        for (int q = 0; q < 2; q++)
            if (gath_rec[q] && !(nsteps == 1 && gath_side[q] == cur)) CK(cudaStreamWaitEvent(st, ev_gath[q], 0));
        CK(cudaMemsetAsync(counters_b.p, 0, sizeof(counters), st));
        if (!timing_open) { CK(cudaEventRecord(ev0, st)); timing_open = true; }
        // tune once, and again only if the batch grew more than 4x since
        if (tune_on && (tuned_n == 0 || N > 4 * tuned_n) && tune_left == 0) {
            tune_left = TUNE_ROUNDS * max_cfg();
            tuned_n = N;
            for (int q = 0; q < NPH; q++)
                for (int c = 0; c < MAXCFG; c++) { tune_ms[q][c] = 0.0; tune_n[q][c] = 0; }
        }
        int remaining = nsteps;
        while (remaining > 0) {
            const bool tuning = tune_left > 0;
            // a tuning chunk runs one step per candidate; otherwise chunks are
            // powers of two so that their graphs are reused
            int K = tuning ? std::min(remaining, max_cfg()) : std::min(remaining, chunk);
            if (!tuning) while (K & (K - 1)) K &= K - 1;
            const int diag_last = (diagnostics && remaining == K) ? 1 : 0;
            int bs[NPH];
            for (int q = 0; q < NPH; q++) bs[q] = blk[q];
            launch_set_int(step_base_b.as<int>(), gbase, st);
            if (tuning) {
                // each tuning step uses the next candidate for every kernel
                for (int k = 0; k < K; k++) {
                    int bk[NPH];
                    for (int q = 0; q < NPH; q++) bk[q] = cfg[q][(tune_step + k) % ncfg[q]];
                    while ((int)kev.size() < NEV * K) {
                        cudaEvent_t e;
                        CK(cudaEventCreate(&e));
                        kev.push_back(e);
                    }
                    TRY(launch_one(cur ^ (k & 1), (diag_last && k == K - 1) ? 1 : 0, k, bk, &kev[NEV * k],
                                   false));
                }
            } else {
                TRY(launch_chunk(K, cur, diag_last, bs, false, phase_every));
            }
            // the steps just launched (directly or as a graph) update the
            // working bond records
            if (prec != GODAR_PREC_FP64 && NB > 0) wdirty = true;
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(h_status, status.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            const int stt = h_status[0];
            if (stt & ST_NAN) { set_err("non-finite floe state"); return GODAR_ERR_NAN; }
            if (stt & ST_ROW_OVERFLOW) { set_err("inconsistent neighbour rows"); return GODAR_ERR_CAPACITY; }
            if (stt & ST_TIMEOUT) { set_err("a device wait gave up; the step did not complete"); return GODAR_ERR_TIMEOUT; }
            int done = K;
            if (stt & ST_EXPIRED) done = std::max(0, std::min(K, h_status[1] - gbase + 1));
            gbase += K;
            const bool conc = concurrent_bonds();
            for (int k = 0; k < done; k++) {
                if (!tuning && !(phase_every > 0 && k % phase_every == 0)) continue;
                phase_steps++;
                const cudaEvent_t *E7 = &kev[NEV * k];
                float tstep = 0.f;
                CK(cudaEventElapsedTime(&tstep, E7[0], E7[5]));
                kernel_ms += tstep;
                for (int q = 0; q < NPH; q++) {
                    float t = 0.f;
                    // the bond kernel, beside the pair kernels, runs from the
                    // step's start to its own event
                    if (q == 2 && conc) CK(cudaEventElapsedTime(&t, E7[0], E7[6]));
                    else CK(cudaEventElapsedTime(&t, E7[q], E7[q + 1]));
                    phase_ms[q] += t;
                    // a candidate's time is its fastest step: the first
                    // step also loads the kernels, and a diagnostic step
                    // does more work, so neither is compared
                    if (tuning && !(diag_last && k == K - 1)) {
                        const int c = (tune_step + k) % ncfg[q];
                        tune_ms[q][c] = tune_n[q][c] ? std::min(tune_ms[q][c], (double)t) : (double)t;
                        tune_n[q][c]++;
                    }
                }
            }
            if (tuning) {
                tune_step += done;
                tune_left = std::max(0, tune_left - done);
                if (tune_left == 0) {
                    for (int q = 0; q < NPH; q++) {
                        int bc = -1;
                        double bt = 0.0;
                        for (int c = 0; c < ncfg[q]; c++) {
                            if (!tune_n[q][c]) continue;
                            const double t = tune_ms[q][c];
                            if (bc < 0 || t < bt) { bc = c; bt = t; }
                        }
                        if (bc >= 0) blk[q] = cfg[q][bc];
                    }
                    if (tune_log) {
                        // each kernel's candidates (block/variant) and the
                        // fastest of their steps, in microseconds
                        for (int q = 0; q < NPH; q++) {
                            fprintf(stderr, "godar tune: kernel %d, %d floes:", q, N);
                            for (int c = 0; c < ncfg[q]; c++)
                                if (tune_n[q][c])
                                    fprintf(stderr, " %d/%d %.1f", cfg_block(cfg[q][c]), cfg_variant(cfg[q][c]),
                                            1e3 * tune_ms[q][c]);
                            fprintf(stderr, " -> %d/%d\n", cfg_block(blk[q]), cfg_variant(blk[q]));
                        }
                    }
                    drop_graphs();
                }
            }
            launches += done;
            kernel_launches += (long long)done * kernels_per_step();
            cur ^= (done & 1);
            remaining -= done;
            for (auto &I : insts) I.steps += done;
            if (stt & ST_EXPIRED) {
                // a rebuild rewrites the other side: the copy must be done
                for (int q = 0; q < 2; q++)
                    if (gath_rec[q]) CK(cudaStreamWaitEvent(st, ev_gath[q], 0));
                TRY(rebuild(nullptr, nullptr, false));
                chunk = std::max(4, chunk / 2);
            } else if (!tuning) {
                chunk = std::min(chunk * 2, 256);
            }
        }
        CK(cudaMemcpyAsync(counters, counters_b.p, sizeof(counters), cudaMemcpyDeviceToHost, st));
        CK(cudaEventRecord(ev1, st));
        CK(cudaStreamSynchronize(st));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ev0, ev1));
        timing_open = false;
        last_ms = ms;
        return GODAR_OK;
    }

    // ----------------------------------------------------------- async steps
    // Launches nsteps time steps and returns without waiting for them: the
    // status of the steps of earlier calls is read once these are queued
    // behind them, so the device always has the next step.  A chunk queued
    // behind one that raised an expiry does nothing (its kernels see the
    // expiry, numbered before their own steps); the host then rebuilds and
    // runs every lost step again, each with the uniform forcing it was
    // launched with.  Falls back to run() while the tuner measures, while a
    // membership change waits or without CUDA graphs.
    int run_async(int nsteps) {
        if (nsteps <= 0) return GODAR_OK;
        const bool tune_due = tune_on && (tuned_n == 0 || N > 4 * tuned_n);
        if (dirty || !have_rows || N == 0 || !graphs_on || tune_left > 0 || tune_due) {
            TRY(resolve());
            return run(nsteps);
        }
        const size_t before = pend.size();
        for (int q = 0; q < 2; q++)
            if (gath_rec[q] && !(nsteps == 1 && gath_side[q] == cur)) CK(cudaStreamWaitEvent(st, ev_gath[q], 0));
        CK(cudaMemsetAsync(counters_b.p, 0, sizeof(counters), st));
        if (!timing_open) { CK(cudaEventRecord(ev0, st)); timing_open = true; }
        int remaining = nsteps;
        while (remaining > 0) {
            if ((int)pend.size() >= RING) TRY(resolve_front(pend.size()));
            int K = std::min(remaining, chunk);
            while (K & (K - 1)) K &= K - 1;
            const int diag_last = (diagnostics && remaining == K) ? 1 : 0;
            Pending P;
            P.base = gbase; P.K = K; P.c0 = cur; P.slot = ring_next;
            P.diag = diag_last != 0;
            P.uvw = cur_uvw;
            ring_next = (ring_next + 1) % RING;
            launch_set_int(step_base_b.as<int>(), gbase, st);
            // queued steps record no timing events: nothing reads them
            TRY(launch_chunk(K, cur, diag_last, blk, false, 0));
            if (prec != GODAR_PREC_FP64 && NB > 0) wdirty = true;
            CK(cudaGetLastError());
            int *hs = h_ring + 4 * P.slot;
            CK(cudaMemcpyAsync(hs, status.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
            CK(cudaEventRecord(ring_ev[P.slot], st));
            pend.push_back(std::move(P));
            cur ^= (K & 1);
            gbase += K;
            remaining -= K;
        }
        return resolve_front(std::min(before, pend.size()));
    }

    // Time steps counted as done.
    void account(int done) {
        launches += done;
        kernel_launches += (long long)done * kernels_per_step();
        for (auto &I : insts) I.steps += done;
    }

    // Reads the status of the n oldest launched chunks, in order.
    int resolve_front(size_t n) {
        while (n > 0 && !pend.empty()) {
            const Pending &P = pend.front();
            CK(cudaEventSynchronize(ring_ev[P.slot]));
            const int stt = h_ring[4 * P.slot];
            if (stt & (ST_NAN | ST_ROW_OVERFLOW | ST_TIMEOUT)) {
                CK(cudaStreamSynchronize(st));
                pend.clear();
                timing_open = false;
                if (stt & ST_NAN) { set_err("non-finite floe state"); return GODAR_ERR_NAN; }
                if (stt & ST_ROW_OVERFLOW) { set_err("inconsistent neighbour rows"); return GODAR_ERR_CAPACITY; }
                set_err("a device wait gave up; the step did not complete");
                return GODAR_ERR_TIMEOUT;
            }
            if (stt & ST_EXPIRED) return redo_after_expiry();
            account(P.K);
            chunk = std::min(chunk * 2, 256);
            pend.pop_front();
            n--;
        }
        return GODAR_OK;
    }

    // The oldest launched chunk raised an expiry: its steps up to the one
    // that raised it are kept; the rest of it and every chunk behind it did
    // nothing.  Rebuilds, then runs those steps again (synchronously), each
    // with the uniform forcing and the diagnostics it was launched with.
    int redo_after_expiry() {
        const Pending &P = pend.front();
        const int done = std::max(0, std::min(P.K, h_ring[4 * P.slot + 1] - P.base + 1));
        CK(cudaStreamSynchronize(st));
        struct Redo { int K; bool diag; std::vector<double> uvw; };
        std::vector<Redo> redo;
        if (P.K > done) redo.push_back({P.K - done, P.diag, P.uvw});
        for (size_t i = 1; i < pend.size(); i++) redo.push_back({pend[i].K, pend[i].diag, pend[i].uvw});
        account(done);
        cur = P.c0 ^ (done & 1);
        pend.clear();
        for (int q = 0; q < 2; q++)
            if (gath_rec[q]) CK(cudaStreamWaitEvent(st, ev_gath[q], 0));
        TRY(rebuild(nullptr, nullptr, false));
        chunk = std::max(4, chunk / 2);
        const std::vector<double> latest = cur_uvw;
        const bool diag_now = diagnostics;
        int rc = GODAR_OK;
        for (auto &r : redo) {
            if (!r.uvw.empty() && r.uvw != cur_uvw) rc = set_uniform_forcing(r.uvw.data());
            diagnostics = r.diag;
            if (rc == GODAR_OK) rc = run(r.K);
            if (rc != GODAR_OK) break;
        }
        diagnostics = diag_now;
        TRY(rc);
        if (!latest.empty() && cur_uvw != latest) TRY(set_uniform_forcing(latest.data()));
        return GODAR_OK;
    }

    // Waits for every launched step (the synchronous calls start with it).
    int resolve() {
        if (pend.empty()) return GODAR_OK;
        TRY(resolve_front(pend.size()));
        CK(cudaMemcpyAsync(counters, counters_b.p, sizeof(counters), cudaMemcpyDeviceToHost, st));
        CK(cudaEventRecord(ev1, st));
        CK(cudaStreamSynchronize(st));
        if (timing_open) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, ev0, ev1));
            last_ms = ms;
            timing_open = false;
        }
        return GODAR_OK;
    }

    // Before a read of the state the last call left: every step but those of
    // a last one-step call must be known good (a later step can only be lost
    // to an expiry raised before it).
    int resolve_for_read() {
        if (pend.size() > 1 || (pend.size() == 1 && pend.front().K > 1)) return resolve();
        return GODAR_OK;
    }

    int get_field(int handle, int field, double *out) {
        if (!out || field < 0 || field >= GODAR_F_COUNT) { set_err("bad field"); return GODAR_ERR_BAD_INPUT; }
        Inst *I = find(handle);
        if (!I) { set_err("unknown instance"); return GODAR_ERR_NOT_FOUND; }
        // other fields' admissions and removals wait for the next step: this
        // field's slots stay valid until then
        if (I->pending) TRY(commit());
        launch_gather_field(views(), cur, 0, I->off, I->n, field, tmp_out.as<double>(), st);
        CK(cudaMemcpyAsync(out, tmp_out.p, (size_t)I->n * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return GODAR_OK;
    }

    int set_uniform_forcing(const double *uvw) {
        if (!uvw) return GODAR_ERR_BAD_INPUT;
        TRY(commit());
        const size_t ni = insts.size();
        if (ni == 0) return GODAR_OK;
        for (size_t k = 0; k < ni; k++) {
            insts[k].prm.ua = uvw[4 * k]; insts[k].prm.va = uvw[4 * k + 1];
            insts[k].prm.uw = uvw[4 * k + 2]; insts[k].prm.vw = uvw[4 * k + 3];
            hparams[k].ua = uvw[4 * k]; hparams[k].va = uvw[4 * k + 1];
            hparams[k].uw = uvw[4 * k + 2]; hparams[k].vw = uvw[4 * k + 3];
        }
        cur_uvw.assign(uvw, uvw + 4 * ni);
        // the upload reads a pinned copy of its own: the caller's buffer may
        // change before a queued copy runs
        const int q = fring_next;
        fring_next = (fring_next + 1) % FRING;
        if (fring_used[q]) CK(cudaEventSynchronize(fring_ev[q]));
        if (fring_cap < 4 * ni) {
            for (int k = 0; k < FRING; k++)
                if (fring_used[k]) CK(cudaEventSynchronize(fring_ev[k]));
            for (int k = 0; k < FRING; k++) {
                if (fring[k]) cudaFreeHost(fring[k]);
                fring[k] = nullptr;
            }
            fring_cap = std::max<size_t>(4 * ni, 2 * fring_cap);
            for (int k = 0; k < FRING; k++) CK(cudaMallocHost(&fring[k], fring_cap * sizeof(double)));
        }
        std::memcpy(fring[q], uvw, 4 * ni * sizeof(double));
        // the four doubles are contiguous in InstParams: one strided copy
        CK(cudaMemcpy2DAsync((char *)params_b.p + offsetof(InstParams, ua), sizeof(InstParams), fring[q],
                             4 * sizeof(double), 4 * sizeof(double), ni, cudaMemcpyHostToDevice, st));
        CK(cudaEventRecord(fring_ev[q], st));
        fring_used[q] = true;
        return GODAR_OK;
    }

    // Waits for the read-back of godar_batch_get_all_async.
    int wait_copy() {
        for (int q = 0; q < 2; q++)
            if (copy_pend[q]) {
                CK(cudaEventSynchronize(ev_copy[q]));
                copy_pend[q] = false;
            }
        return GODAR_OK;
    }

    // Gathers fields of the current state on the read-back stream and copies
    // them to the host without waiting; the next step may run meanwhile (it
    // writes the other side), a later one waits for the copy on the device.
    int get_all_async(int nf, const int *fields, double *const *outs) {
        if (nf < 1 || nf > MAX_ASYNC_FIELDS || !fields || !outs) { set_err("1..4 fields"); return GODAR_ERR_BAD_INPUT; }
        for (int k = 0; k < nf; k++)
            if (!outs[k] || fields[k] < 0 || fields[k] >= GODAR_F_TFX) {
                // diagnostics live in one buffer that the next step rewrites
                set_err("state fields (GODAR_F_X .. GODAR_F_OMEGA) only");
                return GODAR_ERR_BAD_INPUT;
            }
        TRY(resolve_for_read());
        TRY(commit());
        if (N == 0) return wait_copy();
        const int sl = aslot, po = sl ^ 1;
        aslot ^= 1;
        // the slot's previous copy (two calls ago) was waited for by the last
        // call; an interleaved synchronous read may have left it otherwise
        if (copy_pend[sl]) {
            CK(cudaEventSynchronize(ev_copy[sl]));
            copy_pend[sl] = false;
        }
        for (int k = 0; k < nf; k++)
            if (async_tmp[sl][k].bytes < (size_t)N * 8) {
                // growing a buffer synchronises the device: nothing in flight
                TRY(wait_copy());
                TRY(async_tmp[sl][k].ensure((size_t)N * 8, &bytes, &mp));
            }
        CK(cudaEventRecord(ev_state, st));
        CK(cudaStreamWaitEvent(stg, ev_state, 0));
        Views V = views();
        for (int k = 0; k < nf; k++) launch_gather_field(V, cur, -1, 0, N, fields[k], async_tmp[sl][k].as<double>(), stg);
        CK(cudaEventRecord(ev_gath[sl], stg));
        gath_rec[sl] = true;
        gath_side[sl] = cur;
        CK(cudaStreamWaitEvent(stc, ev_gath[sl], 0));
        for (int k = 0; k < nf; k++)
            CK(cudaMemcpyAsync(outs[k], async_tmp[sl][k].p, (size_t)N * 8, cudaMemcpyDeviceToHost, stc));
        CK(cudaEventRecord(ev_copy[sl], stc));
        copy_pend[sl] = true;
        // the previous call's outputs are complete when this call returns
        if (copy_pend[po]) {
            CK(cudaEventSynchronize(ev_copy[po]));
            copy_pend[po] = false;
        }
        return GODAR_OK;
    }

    // Per-instance summary of the current state (momentum, kinetic energy,
    // largest speed) reduced on the read-back stream and copied to the host
    // without waiting, in the same two slots as get_all_async.
    int summary_async(double *out) {
        if (!out) { set_err("null output"); return GODAR_ERR_BAD_INPUT; }
        TRY(resolve_for_read());
        TRY(commit());
        const int ni = (int)insts.size();
        if (N == 0 || ni == 0) return wait_copy();
        const int sl = aslot, po = sl ^ 1;
        aslot ^= 1;
        if (copy_pend[sl]) {
            CK(cudaEventSynchronize(ev_copy[sl]));
            copy_pend[sl] = false;
        }
        const size_t nbytes = (size_t)ni * 4 * sizeof(double);
        if (async_tmp[sl][0].bytes < nbytes) {
            TRY(wait_copy());
            TRY(async_tmp[sl][0].ensure(nbytes, &bytes, &mp));
        }
        CK(cudaEventRecord(ev_state, st));
        CK(cudaStreamWaitEvent(stg, ev_state, 0));
        launch_instance_summary(views(), cur, async_tmp[sl][0].as<double>(), stg);
        CK(cudaGetLastError());
        CK(cudaEventRecord(ev_gath[sl], stg));
        gath_rec[sl] = true;
        gath_side[sl] = cur;
        CK(cudaStreamWaitEvent(stc, ev_gath[sl], 0));
        CK(cudaMemcpyAsync(out, async_tmp[sl][0].p, nbytes, cudaMemcpyDeviceToHost, stc));
        CK(cudaEventRecord(ev_copy[sl], stc));
        copy_pend[sl] = true;
        if (copy_pend[po]) {
            CK(cudaEventSynchronize(ev_copy[po]));
            copy_pend[po] = false;
        }
        return GODAR_OK;
    }

    int get_all(int field, double *out) {
        if (!out || field < 0 || field >= GODAR_F_COUNT) { set_err("bad field"); return GODAR_ERR_BAD_INPUT; }
        TRY(wait_copy());
        TRY(commit());
        if (N == 0) return GODAR_OK;
        Views V = views();
        launch_gather_field(V, cur, -1, 0, N, field, tmp_out.as<double>(), st);
        CK(cudaMemcpyAsync(out, tmp_out.p, (size_t)N * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return GODAR_OK;
    }

    int get_pairs(int handle, int which, int32_t *pi, int32_t *pj, double *val, int cap, int *count) {
        Inst *I = find(handle);
        if (!I) { set_err("unknown instance"); return GODAR_ERR_NOT_FOUND; }
        if (which < 0 || which > 2) { set_err("bad pair list"); return GODAR_ERR_BAD_INPUT; }
        // other fields' admissions and removals wait for the next step: this
        // field's slots stay valid until then
        if (I->pending) TRY(commit());
        if (which == 2) TRY(sync_bonds());
        // count first, then fill
        CK(cudaMemsetAsync(tmp_cnt.p, 0, sizeof(int), st));
        launch_list_pairs(views(), cur, 0, I->off, I->n, which, nullptr, nullptr, nullptr, 0, tmp_cnt.as<int>(), st);
        int total = 0;
        CK(cudaMemcpyAsync(&total, tmp_cnt.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (count) *count = total;
        if (total == 0 || cap <= 0) return GODAR_OK;
        TRY(tmp_i.ensure((size_t)total * 4, &bytes, &mp)); TRY(tmp_j.ensure((size_t)total * 4, &bytes, &mp));
        TRY(tmp_v.ensure((size_t)total * 8, &bytes, &mp));
        CK(cudaMemsetAsync(tmp_cnt.p, 0, sizeof(int), st));
        launch_list_pairs(views(), cur, 0, I->off, I->n, which, tmp_i.as<int>(), tmp_j.as<int>(), tmp_v.as<double>(),
                          total, tmp_cnt.as<int>(), st);
        std::vector<int> hi(total), hj(total);
        std::vector<double> hv(total);
        CK(cudaMemcpyAsync(hi.data(), tmp_i.p, (size_t)total * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(hj.data(), tmp_j.p, (size_t)total * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(hv.data(), tmp_v.p, (size_t)total * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        std::vector<int> ord(total);
        std::iota(ord.begin(), ord.end(), 0);
        std::sort(ord.begin(), ord.end(), [&](int a, int b) { return hi[a] != hi[b] ? hi[a] < hi[b] : hj[a] < hj[b]; });
        const int m = std::min(cap, total);
        for (int k = 0; k < m; k++) {
            if (pi) pi[k] = hi[ord[k]];
            if (pj) pj[k] = hj[ord[k]];
            if (val) val[k] = hv[ord[k]];
        }
        return GODAR_OK;
    }
};

// ====================================================================== C ABI
struct godar_ctx {
    Engine eng;
    godar_params prm{};
    int n = 0;
    int handle = -1;
    bool uploaded = false;
    bool started = false;
    // staged upload until the first step decides fresh/restart
    std::vector<double> x, y, r, h, th, om, u, v, field;
    std::vector<int32_t> bi, bj;
    std::vector<double> dmg;
    std::shared_ptr<RestoreExtra> rx;   // from godar_gpu_restore
    std::vector<char> ck;               // last checkpoint built, valid while ck_at == steps taken
    long long ck_at = -1;
};

struct godar_batch {
    Engine eng;
};

// for the output writer (posts.cu)
namespace godar {
int ctx_floe_count(const godar_ctx *c) { return c ? c->n : 0; }
void set_last_error(const std::string &msg) { g_last_error = msg; }
}  // namespace godar

extern "C" {

const char *godar_gpu_version(void) { return "godar_b200 1.0 (sm_100a)"; }

const char *godar_gpu_errstr(int s)
{
    switch (s) {
    case GODAR_OK: return "ok";
    case GODAR_ERR_CUDA: return "CUDA error";
    case GODAR_ERR_BAD_INPUT: return "bad input";
    case GODAR_ERR_CAPACITY: return "capacity exceeded";
    case GODAR_ERR_NAN: return "non-finite state";
    case GODAR_ERR_TIMEOUT: return "device wait timed out";
    case GODAR_ERR_NOMEM: return "device out of memory";
    case GODAR_ERR_STATE: return "call out of order";
    case GODAR_ERR_BUDGET: return "HBM budget exceeded";
    case GODAR_ERR_NOT_FOUND: return "unknown instance";
    case GODAR_ERR_NO_DEVICE: return "no CUDA device";
    case GODAR_ERR_IO: return "file i/o failed";
    default: return "unknown status";
    }
}

const char *godar_gpu_last_error(void) { return g_last_error.c_str(); }

// Every context call but godar_gpu_step_async and godar_gpu_set_diagnostics
// (read when steps are launched) first waits for the steps still queued and
// reports their errors.
#define GODAR_CTX_RESOLVED(c)                             \
    do {                                                  \
        if (!(c)) return GODAR_ERR_BAD_INPUT;             \
        const int rc_ = (c)->eng.resolve();               \
        if (rc_ != GODAR_OK) return rc_;                  \
    } while (0)

int godar_gpu_params_size(void) { return (int)sizeof(godar_params); }

int godar_gpu_derive_params(godar_params *p)
{
    if (!p) return GODAR_ERR_BAD_INPUT;
    p->pi = 4.0 * std::atan(1.0);
    const double nu = p->poiss_ratio;
    p->ec = p->e_modul / (2.0 * (1.0 - nu * nu));
    p->gc = p->e_modul / ((4.0 * (1.0 - nu)) * (2.0 + nu));
    const double le = std::log(p->rest_coeff);
    p->beta = (10.0 * le) / std::sqrt(le * le + p->pi * p->pi);
    p->sin_lat = std::sin(p->lat);
    return GODAR_OK;
}

int godar_gpu_default_params(godar_params *p)
{
    if (!p) return GODAR_ERR_BAD_INPUT;
    std::memset(p, 0, sizeof(*p));
    p->dynamics = 1; p->slipping = 1; p->thermodyn = 0; p->cohesion = 1; p->ridging = 1; p->shelter = 1;
    p->rtree = 1e3; p->ntree = 1.0; p->dt = 1e-3; p->nt = 1e3; p->comp = 1.0;
    p->Cdair = 3e-1; p->Csair = 5e-4; p->Cdwater = 3e-1; p->Cswater = 2e-3; p->z0w = 3.0e-4;
    p->lat = (double)1.4f;
    p->rhoair = 1.3; p->rhoice = 9e2; p->rhowater = 1026.0;
    p->e_modul = 6e9; p->poiss_ratio = 33e-2; p->friction_coeff = 7e-1; p->rest_coeff = 88e-2; p->sigmanc_crit = 1e6;
    p->eb = 6e9; p->lambda_rb = 8e-1; p->lambda_lb = 1.0; p->sigmatb_crit = 1e5; p->sigmacb_crit = 1e6;
    p->tau_crit = 1e6; p->bond_lim = 1e-2; p->dmax = 9e-1; p->dtd = 1.0; p->dth = 1e5;
    p->nx = 5e3; p->ny = 5e3;
    return godar_gpu_derive_params(p);
}

int godar_gpu_create(const godar_params *p, int n, int precision, godar_ctx **out)
{
    if (!p || !out || n <= 0) { set_err("null params/out or n <= 0"); return GODAR_ERR_BAD_INPUT; }
    if (precision != GODAR_PREC_FP64 && precision != GODAR_PREC_MIXED) { set_err("bad precision"); return GODAR_ERR_BAD_INPUT; }
    auto c = std::make_unique<godar_ctx>();
    TRY(c->eng.init(precision, 0));
    c->prm = *p;
    c->n = n;
    *out = c.release();
    return GODAR_OK;
}

int godar_gpu_upload(godar_ctx *c, const double *x, const double *y, const double *r, const double *h,
                     const double *theta, const double *omega, const double *u, const double *v, int nb,
                     const int32_t *bond_i, const int32_t *bond_j, const double *damage)
{
    GODAR_CTX_RESOLVED(c);
    if (!c || !x || !y || !r || !h) { set_err("null input"); return GODAR_ERR_BAD_INPUT; }
    if (nb < 0 || (nb > 0 && (!bond_i || !bond_j))) { set_err("bad bond lists"); return GODAR_ERR_BAD_INPUT; }
    const int n = c->n;
    // the inputs are checked before anything is replaced: a rejected upload
    // leaves the context as it was
    for (int i = 0; i < n; i++)
        if (!std::isfinite(x[i]) || !std::isfinite(y[i]) || !(r[i] > 0) || !(h[i] > 0)) {
            set_err("non-finite position or non-positive radius/thickness");
            return GODAR_ERR_BAD_INPUT;
        }
    for (int k = 0; k < nb; k++) {
        const double d = damage ? damage[k] : 0.0;
        if (bond_i[k] < 0 || bond_i[k] >= n || bond_j[k] < 0 || bond_j[k] >= n || bond_i[k] == bond_j[k] ||
            !(d >= 0.0 && d <= 1.0)) {
            set_err("bad bond index or damage");
            return GODAR_ERR_BAD_INPUT;
        }
    }
    auto cp = [n](const double *a, std::vector<double> &d) { if (a) d.assign(a, a + n); else d.assign(n, 0.0); };
    cp(x, c->x); cp(y, c->y); cp(r, c->r); cp(h, c->h); cp(theta, c->th); cp(omega, c->om); cp(u, c->u); cp(v, c->v);
    c->bi.assign(bond_i, bond_i + nb); c->bj.assign(bond_j, bond_j + nb);
    if (damage) c->dmg.assign(damage, damage + nb); else c->dmg.assign(nb, 0.0);
    if (c->handle >= 0) { c->eng.remove(c->handle); c->handle = -1; }
    c->rx.reset();
    c->uploaded = true;
    c->started = false;
    return GODAR_OK;
}

int godar_gpu_set_field(godar_ctx *c, const double *field)
{
    if (!c || !field || c->prm.field_nx < 2 || c->prm.field_ny < 2) { set_err("field grid not configured"); return GODAR_ERR_BAD_INPUT; }
    if (c->handle >= 0) { set_err("set the field before the first step"); return GODAR_ERR_STATE; }
    c->field.assign(field, field + (size_t)4 * c->prm.field_nx * c->prm.field_ny);
    return GODAR_OK;
}

// The context's field admitted to its engine at its first step.
static int ctx_admit(godar_ctx *c, int tstep, int restart)
{
    if (!c->uploaded) { set_err("step before upload"); return GODAR_ERR_STATE; }
    if (c->handle < 0) {
        const bool fresh = tstep == 1 && restart != 1 && c->prm.cohesion;
        int hd = -1;
        TRY(c->eng.add(&c->prm, c->n, c->x.data(), c->y.data(), c->r.data(), c->h.data(), c->th.data(),
                       c->om.data(), c->u.data(), c->v.data(), (int)c->bi.size(), c->bi.data(), c->bj.data(),
                       c->dmg.data(), c->field.empty() ? nullptr : c->field.data(), fresh ? 1 : 0, &hd));
        c->handle = hd;
        if (c->rx) {
            TRY(c->eng.attach_restore(hd, c->rx));
            c->rx.reset();
        }
    }
    return GODAR_OK;
}

int godar_gpu_step(godar_ctx *c, int tstep, int restart, int nsteps)
{
    GODAR_CTX_RESOLVED(c);
    if (nsteps < 0) return GODAR_ERR_BAD_INPUT;
    TRY(ctx_admit(c, tstep, restart));
    return c->eng.run(nsteps);
}

int godar_gpu_step_async(godar_ctx *c, int tstep, int restart, int nsteps)
{
    if (!c || nsteps < 0) return GODAR_ERR_BAD_INPUT;
    TRY(ctx_admit(c, tstep, restart));
    return c->eng.run_async(nsteps);
}

int godar_gpu_get_floe_field(godar_ctx *c, int field, double *out)
{
    GODAR_CTX_RESOLVED(c);
    if (!out || field < 0 || field >= GODAR_F_COUNT) { set_err("bad field"); return GODAR_ERR_BAD_INPUT; }
    if (c->handle < 0) {
        if (!c->uploaded) { set_err("no state"); return GODAR_ERR_STATE; }
        if (field >= GODAR_F_TFX) { set_err("diagnostics exist after the first step"); return GODAR_ERR_STATE; }
        const std::vector<double> *src[8] = {&c->x, &c->y, &c->u, &c->v, &c->r, &c->h, &c->th, &c->om};
        std::copy(src[field]->begin(), src[field]->end(), out);
        return GODAR_OK;
    }
    return c->eng.get_field(c->handle, field, out);
}

int godar_gpu_get_pairs(godar_ctx *c, int which, int32_t *pi, int32_t *pj, double *val, int cap, int *count)
{
    GODAR_CTX_RESOLVED(c);
    if (c->handle < 0) { set_err("no step yet"); return GODAR_ERR_STATE; }
    return c->eng.get_pairs(c->handle, which, pi, pj, val, cap, count);
}

int godar_gpu_download(godar_ctx *c, double *const *floe_out, int which, int32_t *pair_i, int32_t *pair_j,
                       double *pair_val, int cap, int *count)
{
    if (!c) return GODAR_ERR_BAD_INPUT;
    if (count) *count = 0;
    if (floe_out)
        for (int f = 0; f < GODAR_F_COUNT; f++)
            if (floe_out[f]) TRY(godar_gpu_get_floe_field(c, f, floe_out[f]));
    if (which >= 0) TRY(godar_gpu_get_pairs(c, which, pair_i, pair_j, pair_val, cap, count));
    return GODAR_OK;
}

int godar_gpu_set_precision(godar_ctx *c, int mode)
{
    GODAR_CTX_RESOLVED(c);
    if (mode != GODAR_PREC_FP64 && mode != GODAR_PREC_MIXED) { set_err("bad precision"); return GODAR_ERR_BAD_INPUT; }
    if (mode == c->eng.prec) return GODAR_OK;
    if (c->handle >= 0) {
        // the two precisions keep different pair histories and bond sides
        set_err("precision is fixed once the field has stepped; create a new context");
        return GODAR_ERR_STATE;
    }
    c->eng.~Engine();
    new (&c->eng) Engine();
    return c->eng.init(mode, 0);
}

int godar_gpu_checkpoint(godar_ctx *c, void *buf, size_t cap, size_t *bytes)
{
    if (!bytes) return GODAR_ERR_BAD_INPUT;
    GODAR_CTX_RESOLVED(c);
    *bytes = 0;
    if (c->handle < 0) { set_err("checkpoint before the first step"); return GODAR_ERR_STATE; }
    if (c->ck_at != c->eng.launches) {
        TRY(c->eng.checkpoint(c->handle, c->ck));
        c->ck_at = c->eng.launches;
    }
    *bytes = c->ck.size();
    if (!buf) return GODAR_OK;
    if (cap < c->ck.size()) { set_err("checkpoint buffer too small"); return GODAR_ERR_CAPACITY; }
    std::memcpy(buf, c->ck.data(), c->ck.size());
    return GODAR_OK;
}

int godar_gpu_restore(godar_ctx *c, const void *buf, size_t size)
{
    GODAR_CTX_RESOLVED(c);
    if (!buf || size < sizeof(CkptHeader)) { set_err("no checkpoint"); return GODAR_ERR_BAD_INPUT; }
    CkptHeader hd;
    std::memcpy(&hd, buf, sizeof(hd));
    if (std::memcmp(hd.magic, "GODARCK1", 8) != 0 || hd.version != 1) { set_err("not a checkpoint"); return GODAR_ERR_BAD_INPUT; }
    if (hd.n != c->n) { set_err("checkpoint of a field of another size"); return GODAR_ERR_BAD_INPUT; }
    if (hd.nb < 0 || hd.nh < 0) { set_err("corrupt checkpoint"); return GODAR_ERR_BAD_INPUT; }
    const size_t n = (size_t)hd.n, nb = (size_t)hd.nb, nh = (size_t)hd.nh;
    const size_t need = sizeof(hd) + 12 * n * 8 + nb * (16 + 80) + nh * (8 + 32);
    if (size != need) { set_err("checkpoint size does not match its header"); return GODAR_ERR_BAD_INPUT; }
    const char *p = (const char *)buf + sizeof(hd);
    auto arr = [&](std::vector<double> &v) { v.resize(n); std::memcpy(v.data(), p, n * 8); p += n * 8; };
    auto rx = std::make_shared<RestoreExtra>();
    arr(c->x); arr(c->y); arr(c->u); arr(c->v); arr(c->r); arr(c->h); arr(c->th); arr(c->om);
    arr(rx->dtb1); arr(rx->dtb2); arr(rx->thb1); arr(rx->thb2);
    HostBonds &B = rx->bonds;
    B.off.assign(n + 1, 0);
    int prev_i = -1, prev_j = -1;
    for (size_t k = 0; k < nb; k++) {
        int32_t ij[4];
        double v[10];
        std::memcpy(ij, p, 16); p += 16;
        std::memcpy(v, p, 80); p += 80;
        const int i = ij[0], j = ij[1];
        if (i < 0 || j <= i || j >= (int)n || i < prev_i || (i == prev_i && j <= prev_j)) {
            set_err("corrupt checkpoint bond list"); return GODAR_ERR_BAD_INPUT;
        }
        prev_i = i; prev_j = j;
        B.off[i + 1]++;
        B.hi.push_back(j); B.flag.push_back(ij[2]);
        B.rb.push_back(v[0]); B.hb.push_back(v[1]); B.lb.push_back(v[2]); B.sb.push_back(v[3]); B.ib.push_back(v[4]);
        B.dnb.push_back(v[5]); B.dtb.push_back(v[6]); B.thji.push_back(v[7]); B.thij.push_back(v[8]);
        B.dmg.push_back(v[9]);
    }
    for (size_t i = 0; i < n; i++) B.off[i + 1] += B.off[i];
    rx->hi.resize(nh); rx->hj.resize(nh); rx->h4.resize(4 * nh);
    for (size_t k = 0; k < nh; k++) {
        int32_t ij[2];
        std::memcpy(ij, p, 8); p += 8;
        std::memcpy(&rx->h4[4 * k], p, 32); p += 32;
        if (ij[0] < 0 || ij[1] <= ij[0] || ij[1] >= (int)n) { set_err("corrupt checkpoint history"); return GODAR_ERR_BAD_INPUT; }
        rx->hi[k] = ij[0]; rx->hj[k] = ij[1];
    }
    for (size_t i = 0; i < n; i++)
        if (!std::isfinite(c->x[i]) || !std::isfinite(c->y[i]) || !(c->r[i] > 0) || !(c->h[i] > 0)) {
            set_err("non-finite position or non-positive radius/thickness"); return GODAR_ERR_BAD_INPUT;
        }
    if (c->handle >= 0) { c->eng.remove(c->handle); c->handle = -1; }
    c->bi.clear(); c->bj.clear(); c->dmg.clear();
    c->rx = rx;
    c->uploaded = true;
    c->started = false;
    return GODAR_OK;
}

int godar_gpu_stats(godar_ctx *c, double *ms, int64_t *counts4)
{
    GODAR_CTX_RESOLVED(c);
    if (ms) *ms = c->eng.last_ms;
    if (counts4) for (int k = 0; k < 4; k++) counts4[k] = (int64_t)c->eng.counters[k];
    return GODAR_OK;
}

void godar_gpu_destroy(godar_ctx *c) { delete c; }

// ---------------------------------------------------------------- batches
int godar_batch_create(int precision, size_t hbm_budget_bytes, godar_batch **out)
{
    if (!out) return GODAR_ERR_BAD_INPUT;
    if (precision != GODAR_PREC_FP64 && precision != GODAR_PREC_MIXED) { set_err("bad precision"); return GODAR_ERR_BAD_INPUT; }
    auto b = std::make_unique<godar_batch>();
    TRY(b->eng.init(precision, hbm_budget_bytes));
    *out = b.release();
    return GODAR_OK;
}

size_t godar_batch_instance_bytes(int n, int nb) { return Engine::instance_bytes(n, nb, GODAR_PREC_FP64); }

int godar_batch_add(godar_batch *b, const godar_params *p, int n, const double *x, const double *y,
                    const double *r, const double *h, const double *theta, const double *omega, const double *u,
                    const double *v, int nb, const int32_t *bond_i, const int32_t *bond_j, const double *damage,
                    const double *field, int restart, int *instance_id)
{
    if (!b) return GODAR_ERR_BAD_INPUT;
    const bool fresh = restart != 1 && p && p->cohesion;
    return b->eng.add(p, n, x, y, r, h, theta, omega, u, v, nb, bond_i, bond_j, damage, field, fresh ? 1 : 0, instance_id);
}

// Every batch call but the queued ones (step_async, set_uniform_forcing,
// summary_async, get_all_async) first waits for the steps still queued and
// reports their errors.
#define GODAR_RESOLVED(b)                                 \
    do {                                                  \
        if (!(b)) return GODAR_ERR_BAD_INPUT;             \
        const int rc_ = (b)->eng.resolve();               \
        if (rc_ != GODAR_OK) return rc_;                  \
    } while (0)

int godar_batch_remove(godar_batch *b, int instance_id)
{
    GODAR_RESOLVED(b);
    return b->eng.remove(instance_id);
}

int godar_batch_step(godar_batch *b, int nsteps)
{
    GODAR_RESOLVED(b);
    return b->eng.run(nsteps);
}

int godar_batch_step_async(godar_batch *b, int nsteps) { return b ? b->eng.run_async(nsteps) : GODAR_ERR_BAD_INPUT; }

int godar_batch_sync(godar_batch *b, double *ms)
{
    GODAR_RESOLVED(b);
    CK(cudaStreamSynchronize(b->eng.st));
    if (ms) *ms = b->eng.last_ms;
    return GODAR_OK;
}

int godar_batch_get_floe_field(godar_batch *b, int instance_id, int field, double *out)
{
    GODAR_RESOLVED(b);
    return b->eng.get_field(instance_id, field, out);
}

int godar_batch_steps_done(godar_batch *b, int instance_id, int64_t *steps)
{
    if (!steps) return GODAR_ERR_BAD_INPUT;
    GODAR_RESOLVED(b);
    Inst *I = b->eng.find(instance_id);
    if (!I) { set_err("unknown instance"); return GODAR_ERR_NOT_FOUND; }
    *steps = I->steps;
    return GODAR_OK;
}

int godar_batch_count(godar_batch *b, int *instances, int64_t *floes)
{
    if (!b) return GODAR_ERR_BAD_INPUT;
    if (instances) *instances = (int)b->eng.insts.size();
    if (floes) { int64_t s = 0; for (auto &I : b->eng.insts) s += I.n; *floes = s; }
    return GODAR_OK;
}

size_t godar_batch_bytes_in_use(godar_batch *b) { return b ? b->eng.bytes.load() : 0; }

int godar_batch_set_uniform_forcing(godar_batch *b, const double *uvw)
{
    return b ? b->eng.set_uniform_forcing(uvw) : GODAR_ERR_BAD_INPUT;
}

int godar_batch_get_all(godar_batch *b, int field, double *out)
{
    GODAR_RESOLVED(b);
    return b->eng.get_all(field, out);
}

int godar_batch_get_all_async(godar_batch *b, int nfields, const int *fields, double *const *outs)
{
    return b ? b->eng.get_all_async(nfields, fields, outs) : GODAR_ERR_BAD_INPUT;
}

int godar_batch_summary_async(godar_batch *b, double *out)
{
    return b ? b->eng.summary_async(out) : GODAR_ERR_BAD_INPUT;
}

int godar_batch_wait(godar_batch *b)
{
    GODAR_RESOLVED(b);
    return b->eng.wait_copy();
}

int godar_batch_phase_stats(godar_batch *b, double *phase_ms, int nphase, int64_t *kernel_launches,
                            int64_t *timed_steps)
{
    if (nphase < 0) return GODAR_ERR_BAD_INPUT;
    GODAR_RESOLVED(b);
    for (int q = 0; q < nphase && phase_ms; q++) phase_ms[q] = q < Engine::NPH ? b->eng.phase_ms[q] : 0.0;
    if (kernel_launches) *kernel_launches = b->eng.kernel_launches;
    if (timed_steps) *timed_steps = b->eng.phase_steps;
    return GODAR_OK;
}

int godar_batch_set_phase_timing(godar_batch *b, int every)
{
    // read when steps are launched: queued steps keep theirs
    if (!b || every < 0) return GODAR_ERR_BAD_INPUT;
    b->eng.phase_every = every;
    return GODAR_OK;
}

int godar_batch_prepare(godar_batch *b, int nsteps)
{
    GODAR_RESOLVED(b);
    return b->eng.prepare(nsteps);
}

int godar_batch_reserve(godar_batch *b, size_t bytes)
{
    GODAR_RESOLVED(b);
    return b->eng.reserve(bytes);
}

int godar_batch_launch_config(godar_batch *b, int *blocks, int nphase, int *graphs_on, int64_t *graph_launches)
{
    if (nphase < 0) return GODAR_ERR_BAD_INPUT;
    GODAR_RESOLVED(b);
    for (int q = 0; q < nphase && blocks; q++) blocks[q] = q < Engine::NPH ? b->eng.blk[q] : 0;
    if (graphs_on) *graphs_on = b->eng.graphs_on ? 1 : 0;
    if (graph_launches) *graph_launches = b->eng.graph_launches;
    return GODAR_OK;
}

int godar_batch_stats(godar_batch *b, double *kernel_ms, int64_t *launches, int64_t *rebuilds, int64_t *counts4)
{
    GODAR_RESOLVED(b);
    if (kernel_ms) *kernel_ms = b->eng.kernel_ms;
    if (launches) *launches = b->eng.launches;
    if (rebuilds) *rebuilds = b->eng.rebuilds;
    if (counts4) for (int k = 0; k < 4; k++) counts4[k] = (int64_t)b->eng.counters[k];
    return GODAR_OK;
}

int godar_batch_set_diagnostics(godar_batch *b, int on)
{
    // read when steps are launched: queued steps keep theirs
    if (!b) return GODAR_ERR_BAD_INPUT;
    b->eng.diagnostics = on != 0;
    return GODAR_OK;
}

int godar_gpu_set_diagnostics(godar_ctx *c, int on)
{
    if (!c) return GODAR_ERR_BAD_INPUT;
    c->eng.diagnostics = on != 0;
    return GODAR_OK;
}

int godar_batch_rebuild_stats(godar_batch *b, double *rebuild_ms, int64_t *rebuilds, int64_t *pairs,
                              int64_t *contact_list)
{
    GODAR_RESOLVED(b);
    if (rebuild_ms) *rebuild_ms = b->eng.rebuild_ms;
    if (rebuilds) *rebuilds = b->eng.rebuilds;
    if (pairs) *pairs = b->eng.E;
    if (contact_list) *contact_list = b->eng.Ec;
    return GODAR_OK;
}

void godar_batch_destroy(godar_batch *b) { delete b; }

}  // extern "C"
