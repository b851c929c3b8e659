// gci_api.cu -- C ABI and host runtime of the integral-direct two-step
// Cholesky decomposition of (pq|rs) and the AO->MO transformation.
//
// Control flow follows the reference driver (TwoStepCholesky*.f90,
// Cholesky_Gammcor.f90); the integral, pivot-search and contraction work
// runs on the device (eri_kernels.cu and the Hermite-matrix kernels for the
// integrals, chol_kernels.cu for the pivot search, dense_fp64.cu for the FP64
// GEMMs, triangular solves and the V_JJ factorisation, ozaki_gemm.cu for the
// split-precision int8 tensor-core GEMMs).  No vendor BLAS or solver library.
#include "../../include/gci.h"
#include "gci_common.h"
#include "gci_runtime.h"
#include "host_math.h"
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace gci {

// ------------------------------------------------------------------ errors
static thread_local std::string g_last_error;
struct Failure {
    int code;
    std::string msg;
};
[[noreturn]] static void fail(int code, const std::string& msg) { throw Failure{code, msg}; }
#define CU(x)                                                                                   \
    do {                                                                                        \
        cudaError_t e_ = (x);                                                                   \
        if (e_ != cudaSuccess) fail(GCI_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <class F>
static int guarded(F&& f)
{
    try {
        f();
        return GCI_OK;
    } catch (const Failure& e) {
        g_last_error = e.msg;
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return GCI_ERR_NOMEM;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return GCI_ERR_ARG;
    }
}

// ------------------------------------------------------------------ launch counter
static std::atomic<int64_t> g_launches{0};
void count_launch(int64_t n) { g_launches += n; }
int64_t launches() { return g_launches.load(); }

// ------------------------------------------------------------------ device buffers
// Stream of the calling thread's current context (set by ctx()).  Device
// buffers are allocated and freed stream-ordered on it, so that a free does
// not synchronise the whole device while other streams (the workers of a
// batch) are running.
static thread_local cudaStream_t t_stream = nullptr;
// The library's own memory pool.  Freed blocks stay mapped for the rest of a
// call (mapping device memory costs more than the kernels of a small molecule,
// and re-mapping the multi-GB Cholesky buffers inside the stream would stall
// it); when a top-level call returns, the pool is trimmed to kPoolKeepBytes.
// The pool is created with the process-wide context.
static cudaMemPool_t g_mempool = nullptr;
constexpr uint64_t kPoolKeepBytes = (uint64_t)8 << 30;

static void pool_trim()
{
    if (g_mempool) cudaMemPoolTrimTo(g_mempool, (size_t)kPoolKeepBytes);
}

template <class T>
struct DVec {
    T* p = nullptr;
    size_t n = 0;
    DVec() = default;
    DVec(const DVec&) = delete;
    DVec& operator=(const DVec&) = delete;
    DVec(DVec&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DVec& operator=(DVec&& o) noexcept
    {
        if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DVec() { release(); }
    void release()
    {
        if (p) cudaFreeAsync(p, t_stream);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count)
    {
        if (count == n && p) return;
        release();
        if (count == 0) return;
        cudaError_t e = g_mempool ? cudaMallocFromPoolAsync((void**)&p, count * sizeof(T), g_mempool, t_stream)
                                  : cudaMallocAsync((void**)&p, count * sizeof(T), t_stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            fail(GCI_ERR_NOMEM, "device allocation of " + std::to_string(count * sizeof(T)) + " bytes failed");
        }
        n = count;
    }
    void ensure(size_t count)
    {
        if (count > n) alloc(count);
    }
    void upload(const std::vector<T>& h, cudaStream_t s)
    {
        ensure(h.size() ? h.size() : 1);
        if (!h.empty()) CU(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    }
};

// ------------------------------------------------------------------ context
constexpr int kAuxStreams = 4;
struct Context {
    std::atomic<bool> ready{false};
    int device = 0;
    cudaStream_t stream = nullptr;
    // streams on which independent class launches of one ERI stage overlap
    // (forked from and joined back into `stream` by events), created on first use
    cudaStream_t aux[kAuxStreams] = {};
    cudaEvent_t ev_fork = nullptr;
    cudaEvent_t ev_join[kAuxStreams] = {};
    DVec<double> boys;
    DVec<int> err;
};
static Context g_ctx;
// Worker contexts of gci_rkpq_batch (own stream and error word each; the Boys
// table is g_ctx's), kept for the process.
static std::vector<std::unique_ptr<Context>> g_pool;
// Context of a batch worker thread; nullptr: the process-wide g_ctx.
static thread_local Context* t_cur = nullptr;

static void context_streams(Context& c)
{
    CU(cudaGetDevice(&c.device));
    CU(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
}

static Context& ctx()
{
    if (t_cur) {
        t_stream = t_cur->stream;
        return *t_cur;
    }
    // the process-wide context is created once; concurrent first calls wait here
    static std::mutex init_mutex;
    std::unique_lock<std::mutex> init_lock(init_mutex, std::defer_lock);
    if (!g_ctx.ready) init_lock.lock();
    if (!g_ctx.ready) {
        int ndev = 0;
        cudaError_t e = cudaGetDeviceCount(&ndev);
        if (e != cudaSuccess || ndev == 0) fail(GCI_ERR_CUDA, "no CUDA device available");
        context_streams(g_ctx);
        t_stream = g_ctx.stream;
        if (!g_mempool) {
            cudaMemPoolProps props = {};
            props.allocType = cudaMemAllocationTypePinned;
            props.handleTypes = cudaMemHandleTypeNone;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = g_ctx.device;
            CU(cudaMemPoolCreate(&g_mempool, &props));
            uint64_t keep = ~(uint64_t)0;   // no release at synchronisation; pool_trim() after each call
            CU(cudaMemPoolSetAttribute(g_mempool, cudaMemPoolAttrReleaseThreshold, &keep));
        }
        CU(eri_module_init());
        std::vector<double> tab = boys_table(kBoysMaxM);
        g_ctx.boys.upload(tab, g_ctx.stream);
        g_ctx.err.alloc(1);
        CU(cudaMemsetAsync(g_ctx.err.p, 0, sizeof(int), g_ctx.stream));
        CU(cudaStreamSynchronize(g_ctx.stream));
        g_ctx.ready = true;
    }
    t_stream = g_ctx.stream;
    return g_ctx;
}

// The first n worker contexts, created on first use (calling thread, after g_ctx).
static void ensure_pool(int n)
{
    Context& M = ctx();
    while ((int)g_pool.size() < n) {
        std::unique_ptr<Context> c(new Context());
        context_streams(*c);
        t_stream = c->stream;
        c->err.alloc(1);
        CU(cudaMemsetAsync(c->err.p, 0, sizeof(int), c->stream));
        CU(cudaStreamSynchronize(c->stream));
        c->ready = true;
        g_pool.push_back(std::move(c));
    }
    t_stream = M.stream;
}

// ------------------------------------------------------------------ phase timer
enum Phase { kVdiag = 0, kStep1Eri, kSubtractR, kPivots, kCompress, kVjjEri, kPotrf, kFullEri, kInvLGemm, kMoGemm, kNumPhases };
struct PhaseTimer {
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
    double acc[kNumPhases] = {0};
    cudaEvent_t cur_start = nullptr;
    int cur = -1;
    cudaStream_t s = nullptr;
    void start(int ph)
    {
        cudaEvent_t e;
        CU(cudaEventCreate(&e));
        CU(cudaEventRecord(e, s));
        cur_start = e;
        cur = ph;
    }
    void stop()
    {
        cudaEvent_t e;
        CU(cudaEventCreate(&e));
        CU(cudaEventRecord(e, s));
        pending.push_back({cur, {cur_start, e}});
        cur = -1;
    }
    void flush()
    {
        for (auto& p : pending) {
            float ms = 0.f;
            CU(cudaEventSynchronize(p.second.second));
            CU(cudaEventElapsedTime(&ms, p.second.first, p.second.second));
            acc[p.first] += ms * 1e-3;
            cudaEventDestroy(p.second.first);
            cudaEventDestroy(p.second.second);
        }
        pending.clear();
    }
};

// ------------------------------------------------------------------ basis + pairs
struct HostBasis {
    int nsh = 0, spher = 1, lmax = 0;
    int64_t nao = 0;
    std::vector<double> xyz, exps, coefs, tmat;
    std::vector<int> L, nprim, poff, nfunc, loc, toff, atom;
};

static HostBasis make_basis(const gci_basis* b)
{
    if (!b) fail(GCI_ERR_ARG, "basis is NULL");
    if (b->nshells <= 0 || b->natoms <= 0 || b->nshellparams <= 0) fail(GCI_ERR_ARG, "empty basis");
    HostBasis h;
    h.nsh = (int)b->nshells;
    h.spher = b->spher_ao ? 1 : 0;
    h.xyz.resize(3 * h.nsh);
    h.L.resize(h.nsh); h.nprim.resize(h.nsh); h.poff.resize(h.nsh); h.nfunc.resize(h.nsh);
    h.loc.resize(h.nsh); h.toff.resize(h.nsh); h.atom.resize(h.nsh);
    for (int s = 0; s < h.nsh; ++s) {
        const int64_t at = b->shell_centers[s] - 1, pr = b->shell_params_idx[s] - 1;
        if (at < 0 || at >= b->natoms) fail(GCI_ERR_ARG, "shell centre index out of range");
        if (pr < 0 || pr >= b->nshellparams) fail(GCI_ERR_ARG, "shell parameter index out of range");
        const int l = (int)b->shell_momentum[pr];
        const int np = (int)b->nprimitives[pr];
        if (l < 0) fail(GCI_ERR_ARG, "negative angular momentum");
        if (l > kMaxL)
            fail(GCI_ERR_UNSUPPORTED, "Basis set includes angular momenta unsupported by the GPU ERI kernels (l > " +
                                          std::to_string(kMaxL) + ")");
        if (np <= 0 || np > b->ldprim) fail(GCI_ERR_ARG, "invalid number of primitives");
        h.atom[s] = (int)at;
        for (int k = 0; k < 3; ++k) h.xyz[3 * s + k] = b->atom_coords[3 * at + k];
        h.L[s] = l;
        h.lmax = std::max(h.lmax, l);
        h.nprim[s] = np;
        h.poff[s] = (int)h.exps.size();
        for (int i = 0; i < np; ++i) {
            h.exps.push_back(b->exponents[pr * b->ldprim + i]);
            h.coefs.push_back(b->cntr_coeffs[pr * b->ldprim + i]);
        }
        const int nc = ncart(l);
        const int nf = h.spher ? 2 * l + 1 : nc;
        if (nf > b->ldnorm) fail(GCI_ERR_ARG, "norm_factors leading dimension too small");
        h.nfunc[s] = nf;
        h.loc[s] = (int)h.nao;
        h.nao += nf;
        h.toff[s] = (int)h.tmat.size();
        std::vector<double> U((size_t)nc * nc, 0.0);
        if (h.spher) spher_coeffs(l, U.data());
        const double* nrm = b->norm_factors + pr * b->ldnorm;
        for (int m = 0; m < nf; ++m)
            for (int c = 0; c < nc; ++c) {
                double v;
                if (h.spher) v = nrm[m] * U[m * nc + c];
                else v = (m == c) ? nrm[m] : 0.0;
                h.tmat.push_back(v);
            }
    }
    return h;
}

struct DevBasis {
    DVec<double> xyz, exps, coefs, tmat;
    DVec<int> poff, nfunc, loc, toff;
};

struct PairTable {
    int64_t n = 0;
    std::vector<int> A, B, type, dim, nab;    // stored A >= B; dim = orbital pairs kept; nab = Na*Nb
    std::vector<int64_t> vdloc;                 // offsets in the Vdiag order
    std::vector<ShellPairDev> h;
    DVec<ShellPairDev> d;
    DVec<double> pp;
    DVec<int> plist;
};

static int64_t pair_local(int a, int b, int Na, bool same)
{
    if (!same) return a + (int64_t)Na * b;
    if (a < b) return -1;
    return (int64_t)b * Na - (int64_t)b * (b - 1) / 2 + (a - b);
}

// ------------------------------------------------------------------ ERI stage dispatch
struct PairMap {
    std::vector<int64_t> off;
    std::vector<int> map;
    DVec<int64_t> doff;
    DVec<int> dmap;
    void reset(int64_t npairs)
    {
        off.assign(npairs, -1);
        map.clear();
    }
    // append an entry block for pair `id` of Na*Nb slots
    int* add(int id, int nab)
    {
        off[id] = (int64_t)map.size();
        map.resize(map.size() + nab, -1);
        return map.data() + off[id];
    }
    void upload(cudaStream_t s)
    {
        for (auto& o : off) if (o < 0) o = 0;
        doff.upload(off, s);
        if (map.empty()) map.push_back(-1);
        dmap.upload(map, s);
    }
};

enum GemmPhase { kGemmSubtractR = 0, kGemmLnew, kGemmPotrf, kGemmInvL, kGemmMo, kNumGemm };

struct Handle;
static void run_eri(Handle& H, const std::vector<int>& bra, const std::vector<int>& ket, int mode, PairMap* rows,
                    PairMap* cols, double* out, int64_t ldo, int64_t jcount = 0);

struct Handle {
    HostBasis hb;
    DevBasis db;
    PairTable pt;
    double tau = 1e-6, kappa = 0.0;
    int flags = 0;
    // results of step 1 (0-based)
    int64_t nsp = 0, npq = 0, nvecs = 0, nsubsets = 0, msd = 0, npsp = 0;
    std::vector<int> bsp;                  // BASE pair ids (all-pair index) in BASE order
    std::vector<int64_t> fullloc, subloc, subidx;
    std::vector<int64_t> subsetdim, subsetlo, subsethi;
    std::vector<int> pivots;
    std::vector<int64_t> pivot_order;
    std::vector<double> pivot_dmax;
    std::vector<int> psp, pspdim, porb;    // pivot shell pairs (BASE index), dims, orbital pair (full block)
    std::vector<int64_t> psploc;
    int converged = 0;
    int64_t nmacro = 0;
    DVec<double> invl;                     // nvecs x nvecs
    DVec<double> rkpq;                     // nvecs x msd x nsubsets (if materialised)
    bool have_rkpq = false;
    PairMap pivmap;                        // pivot columns, by pair id
    PhaseTimer timer;
    double t_rkpq = 0.0, t_rkab = 0.0;
    // work counters: GEMM flops per phase and ERI work per canonical class
    double gemm_flops[kNumGemm] = {0};
    // per canonical class: quartets, primitive quartets after the pair screen, integrals, primitive
    // quartets before it, bra primitive pairs x quartets, ket primitive pairs x quartets
    static constexpr int kNumStats = 6;
    double eri_stats[kNumPairTypes][kNumPairTypes][kNumStats] = {};
    // scratch reused across ERI launches
    DVec<int> d_bra, d_ket;
    // Hermite-matrix path: row vectors of every pair that entered a product
    // stage (offsets by pair id, -1 = not built) and the per-call column data
    std::vector<int64_t> hm_rowoff_h;
    DVec<int64_t> hm_rowoff;
    DVec<double> hm_rowvec;
    DVec<int> hm_ids;
    DVec<HmChunk> hm_chunks;
    DVec<int> hm_colfun, hm_colout, hm_chunkids;
    DVec<double> hm_colvec;
    DVec<unsigned long long> hm_counters;
    double hm_flops = 0.0;
    // per Hermite-matrix class (L1, L2, column tiles): launches, device seconds
    // (profiling mode only) and DMMA flops issued
    double hm_class[kMaxPairL + 1][kMaxPairL + 1][kHmMaxNT][3] = {};                 // DMMA arithmetic issued by the Hermite-matrix kernels (padding included)
};

// Primitive pairs whose weight |c_a c_b| K_ab (pi/P)^{3/2} (1+|PA|)^la (1+|PB|)^lb is
// below kPrimRel of the largest in the shell pair, or below kPrimAbs, are not
// stored: their share of any integral is below the FP64 rounding level.  The
// reference evaluates every primitive quartet; the difference is < 1e-15 relative.
static constexpr double kPrimRel = 1.0e-17;
static constexpr double kPrimAbs = 1.0e-22;

// Host half of the pair table: every shell pair A >= B in the Vdiag order with
// its orientation, kept primitive pairs (plist) and record offsets; `rec` is
// the total size of the primitive-pair records in doubles.
static void build_pair_table(const HostBasis& b, PairTable& P, std::vector<int>& plist, int64_t& rec_total)
{
    const int nsh = b.nsh;
    P.n = (int64_t)nsh * (nsh + 1) / 2;
    P.A.resize(P.n); P.B.resize(P.n); P.type.resize(P.n); P.dim.resize(P.n); P.nab.resize(P.n);
    P.vdloc.resize(P.n); P.h.resize(P.n);
    std::vector<double> w;
    std::vector<double> minexp(nsh, 1e300);
    for (int s = 0; s < nsh; ++s)
        for (int i = 0; i < b.nprim[s]; ++i) minexp[s] = std::min(minexp[s], b.exps[b.poff[s] + i]);
    int64_t sp = 0, loc = 0, rec = 0;
    for (int B = 0; B < nsh; ++B)
        for (int A = B; A < nsh; ++A) {
            const int Na = b.nfunc[A], Nb = b.nfunc[B];
            P.A[sp] = A; P.B[sp] = B;
            P.nab[sp] = Na * Nb;
            P.dim[sp] = (A != B) ? Na * Nb : Na * (Na + 1) / 2;
            P.vdloc[sp] = loc;
            loc += P.dim[sp];
            ShellPairDev d{};
            // canonical orientation: higher l first (as the reference's frontends);
            // for equal l the tighter shell (larger smallest exponent) is the origin of
            // the horizontal recurrence, which keeps its cancellation bounded
            bool sw = b.L[A] < b.L[B];
            if (b.L[A] == b.L[B] && A != B) sw = minexp[A] < minexp[B];
            d.s1 = sw ? B : A;
            d.s2 = sw ? A : B;
            d.swap = sw ? 1 : 0;
            d.l1 = b.L[d.s1];
            d.l2 = b.L[d.s2];
            d.nprim1 = b.nprim[d.s1];
            d.nprim2 = b.nprim[d.s2];
            const double* ra = &b.xyz[3 * d.s1];
            const double* rb = &b.xyz[3 * d.s2];
            const double r2 = (ra[0] - rb[0]) * (ra[0] - rb[0]) + (ra[1] - rb[1]) * (ra[1] - rb[1]) +
                              (ra[2] - rb[2]) * (ra[2] - rb[2]);
            const double r = std::sqrt(r2);
            w.assign((size_t)d.nprim1 * d.nprim2, 0.0);
            double wmax = 0.0;
            for (int gb = 0; gb < d.nprim2; ++gb)
                for (int ga = 0; ga < d.nprim1; ++ga) {
                    const double ea = b.exps[b.poff[d.s1] + ga], eb = b.exps[b.poff[d.s2] + gb];
                    const double ca = b.coefs[b.poff[d.s1] + ga], cb = b.coefs[b.poff[d.s2] + gb];
                    const double p = ea + eb;
                    const double kab = std::exp(-ea * eb / p * r2);
                    const double pa = eb / p * r, pbd = ea / p * r;   // |P - A|, |P - B|
                    const double v = std::fabs(ca * cb) * kab * std::pow(kPi / p, 1.5) *
                                     std::pow(1.0 + pa, d.l1) * std::pow(1.0 + pbd, d.l2);
                    w[ga + (size_t)d.nprim1 * gb] = v;
                    wmax = std::max(wmax, v);
                }
            d.list_off = (int64_t)plist.size();
            int kept = 0;
            for (int gb = 0; gb < d.nprim2; ++gb)
                for (int ga = 0; ga < d.nprim1; ++ga) {
                    const double v = w[ga + (size_t)d.nprim1 * gb];
                    if (v >= kPrimAbs && v >= kPrimRel * wmax) {
                        plist.push_back(ga | (gb << 8));
                        ++kept;
                    }
                }
            d.npp = kept;
            d.rec_off = rec;
            rec += (int64_t)kept * pp_record(d.l1, d.l2);
            P.type[sp] = pair_type(d.l1, d.l2);
            P.h[sp] = d;
            ++sp;
        }
    rec_total = rec;
}

static void setup_pairs(Handle& H)
{
    Context& C = ctx();
    const HostBasis& b = H.hb;
    PairTable& P = H.pt;
    std::vector<int> plist;
    int64_t rec = 0;
    build_pair_table(b, P, plist, rec);
    DevBasis& D = H.db;
    D.xyz.upload(b.xyz, C.stream);
    D.exps.upload(b.exps, C.stream);
    D.coefs.upload(b.coefs, C.stream);
    D.tmat.upload(b.tmat, C.stream);
    D.poff.upload(b.poff, C.stream);
    D.nfunc.upload(b.nfunc, C.stream);
    D.loc.upload(b.loc, C.stream);
    D.toff.upload(b.toff, C.stream);
    P.d.upload(P.h, C.stream);
    if (plist.empty()) plist.push_back(0);
    P.plist.upload(plist, C.stream);
    P.pp.alloc(rec > 0 ? rec : 1);
    CU(pair_records_launch(P.d.p, (int)P.n, D.xyz.p, D.poff.p, D.exps.p, D.coefs.p, P.plist.p, P.pp.p, C.stream));
}

// Hermite-matrix path switch (gci_eri_hm); used for spherical bases in the
// product and dense modes.
static std::atomic<int> g_hm_enabled{1};
// profiling mode (gci_eri_hm(2)): class launches run one after another on the
// context stream, each bracketed by events, and their times are kept per class
static std::atomic<int> g_hm_profile{0};

// Row vectors of `ids` (and of every pair built before) in H.hm_rowvec.
static void hm_ensure_rows(Handle& H, const std::vector<int>& ids)
{
    Context& C = ctx();
    const PairTable& P = H.pt;
    if ((int64_t)H.hm_rowoff_h.size() != P.n) H.hm_rowoff_h.assign(P.n, -1);
    bool missing = false;
    for (int id : ids)
        if (H.hm_rowoff_h[id] < 0) { missing = true; break; }
    if (!missing) return;
    std::vector<char> want(P.n, 0);
    for (int64_t id = 0; id < P.n; ++id) want[id] = H.hm_rowoff_h[id] >= 0;
    for (int id : ids) want[id] = 1;
    std::vector<int> list;
    std::vector<int64_t> off(P.n, 0);
    int64_t tot = 0;
    for (int64_t id = 0; id < P.n; ++id) {
        if (!want[id]) continue;
        list.push_back((int)id);
        off[id] = tot;
        tot += (int64_t)P.h[id].npp * hm_row_stride(P.h[id].l1 + P.h[id].l2);
    }
    H.hm_rowvec.alloc((size_t)std::max<int64_t>(tot, 1));
    H.hm_rowoff.upload(off, C.stream);
    H.hm_ids.upload(list, C.stream);
    CU(hm_rowvec_launch(H.hm_ids.p, (int)list.size(), P.d.p, P.pp.p, H.hm_rowoff.p, H.db.tmat.p, H.db.toff.p,
                        H.db.nfunc.p, H.hm_rowvec.p, C.stream));
    for (int64_t id = 0; id < P.n; ++id) H.hm_rowoff_h[id] = want[id] ? off[id] : -1;
}

// Product / dense stage on the Hermite-matrix kernels.  gb/sb: row pairs
// grouped by pair type (already on the device in H.d_bra); gk/sk: column
// pairs grouped by type; `cols` gives the requested columns of each column
// pair (entries >= 0) and their output column or j index.
static void run_eri_hm(Handle& H, const std::vector<int>& gb, const std::vector<int64_t>& sb,
                       const std::vector<int>& gk, const std::vector<int64_t>& sk, int mode, PairMap* rows,
                       PairMap* cols, double* out, int64_t ldo, int64_t jcount)
{
    Context& C = ctx();
    const PairTable& P = H.pt;
    hm_ensure_rows(H, gb);
    // column chunks, one set per chunk width in use: rows of level L1 take chunks of at
    // most 8 hm_max_nt(L1) columns; within a set, grouped by (column type, tiles)
    bool width_used[kHmMaxNT + 1] = {};
    for (int tb = 0; tb < kNumPairTypes; ++tb)
        if (sb[tb + 1] > sb[tb]) width_used[hm_max_nt(type_lsum(tb))] = true;
    std::vector<HmChunk> chunks;
    std::vector<int> colfun, colout;
    auto gidx = [](int w, int tk, int nt) { return ((size_t)w * kNumPairTypes + tk) * kHmMaxNT + nt - 1; };
    std::vector<std::vector<int>> group((size_t)(kHmMaxNT + 1) * kNumPairTypes * kHmMaxNT);
    int64_t voff = 0;
    std::vector<int> fl, ol;
    for (int w = 1; w <= kHmMaxNT; ++w) {
        if (!width_used[w]) continue;
        for (int tk = 0; tk < kNumPairTypes; ++tk)
            for (int64_t q = sk[tk]; q < sk[tk + 1]; ++q) {
                const int id = gk[q];
                const int nab = P.nab[id];
                const int* m = cols->map.data() + cols->off[id];
                fl.clear(); ol.clear();
                for (int f = 0; f < nab; ++f)
                    if (m[f] >= 0) { fl.push_back(f); ol.push_back(m[f]); }
                const int n = (int)fl.size();
                if (n == 0) continue;
                const int nch = (n + 8 * w - 1) / (8 * w);
                const ShellPairDev& d = P.h[id];
                const int L = d.l1 + d.l2;
                for (int c = 0, beg = 0; c < nch; ++c) {
                    const int cnt = n / nch + (c < n % nch ? 1 : 0);
                    HmChunk ch{};
                    ch.pair = id;
                    ch.ncol = cnt;
                    ch.nt = (cnt + 7) / 8;
                    ch.vec_off = voff;
                    ch.col_off = (int64_t)colfun.size();
                    voff += (int64_t)d.npp * hm_col_stride(L, ch.nt);
                    for (int j = beg; j < beg + cnt; ++j) { colfun.push_back(fl[j]); colout.push_back(ol[j]); }
                    beg += cnt;
                    group[gidx(w, tk, ch.nt)].push_back((int)chunks.size());
                    chunks.push_back(ch);
                }
            }
    }
    if (chunks.empty()) return;
    std::vector<int> order;
    std::vector<int64_t> gstart(group.size() + 1, 0);
    for (size_t g = 0; g < group.size(); ++g) {
        gstart[g] = (int64_t)order.size();
        order.insert(order.end(), group[g].begin(), group[g].end());
    }
    gstart[group.size()] = (int64_t)order.size();
    H.hm_chunks.upload(chunks, C.stream);
    H.hm_colfun.upload(colfun, C.stream);
    H.hm_colout.upload(colout, C.stream);
    H.hm_chunkids.upload(order, C.stream);
    H.hm_colvec.ensure((size_t)std::max<int64_t>(voff, 1));
    CU(hm_colvec_launch(H.hm_chunks.p, (int)chunks.size(), P.d.p, P.pp.p, H.hm_colfun.p, H.db.tmat.p, H.db.toff.p,
                        H.db.nfunc.p, H.hm_colvec.p, C.stream));
    HmArgs a{};
    a.pairs = P.d.p;
    a.pp = P.pp.p;
    a.rowvec = H.hm_rowvec.p;
    a.rowvec_off = H.hm_rowoff.p;
    a.chunks = H.hm_chunks.p;
    a.colvec = H.hm_colvec.p;
    a.colout = H.hm_colout.p;
    a.mode = mode;
    a.out = out;
    a.ldo = ldo;
    a.row_off = rows ? rows->doff.p : nullptr;
    a.row_map = rows ? rows->dmap.p : nullptr;
    a.sh_nfunc = H.db.nfunc.p;
    a.sh_loc = H.db.loc.p;
    a.nao = H.hb.nao;
    a.jcount = jcount;
    a.kappa = H.kappa;
    a.boys = g_ctx.boys.p;
    // one task counter per launch
    int64_t nlaunch = 0;
    for (int tb = 0; tb < kNumPairTypes; ++tb)
        if (sb[tb + 1] > sb[tb]) {
            const int w = hm_max_nt(type_lsum(tb));
            for (int tk = 0; tk < kNumPairTypes; ++tk)
                for (int nt = 1; nt <= w; ++nt) nlaunch += gstart[gidx(w, tk, nt) + 1] > gstart[gidx(w, tk, nt)] ? 1 : 0;
        }
    if (nlaunch == 0) return;
    H.hm_counters.ensure((size_t)nlaunch);
    CU(cudaMemsetAsync(H.hm_counters.p, 0, sizeof(unsigned long long) * nlaunch, C.stream));
    // the class launches are independent (disjoint outputs): fork them over the auxiliary streams
    if (!C.ev_fork) {
        CU(cudaEventCreateWithFlags(&C.ev_fork, cudaEventDisableTiming));
        for (int q = 0; q < kAuxStreams; ++q) {
            CU(cudaStreamCreateWithFlags(&C.aux[q], cudaStreamNonBlocking));
            CU(cudaEventCreateWithFlags(&C.ev_join[q], cudaEventDisableTiming));
        }
    }
    CU(cudaEventRecord(C.ev_fork, C.stream));
    for (int q = 0; q < kAuxStreams; ++q) CU(cudaStreamWaitEvent(C.aux[q], C.ev_fork, 0));
    const bool prof = g_hm_profile.load() != 0;
    std::vector<std::pair<double*, std::pair<cudaEvent_t, cudaEvent_t>>> timed;
    int64_t li = 0;
    for (int tb = 0; tb < kNumPairTypes; ++tb) {
        const int64_t nb = sb[tb + 1] - sb[tb];
        if (nb == 0) continue;
        const int L1 = type_lsum(tb);
        double npb = 0.0, rowt = 0.0;
        for (int64_t q = sb[tb]; q < sb[tb + 1]; ++q) {
            const int id = gb[q];
            npb += P.h[id].npp;
            rowt += (double)P.h[id].npp * ((P.nab[id] + 7) / 8);
        }
        const int w = hm_max_nt(L1);
        for (int tk = 0; tk < kNumPairTypes; ++tk)
            for (int nt = 1; nt <= w; ++nt) {
                const size_t g = gidx(w, tk, nt);
                const int64_t nc = gstart[g + 1] - gstart[g];
                if (nc == 0) continue;
                const int L2 = type_lsum(tk);
                double npk = 0.0;
                for (int64_t q = gstart[g]; q < gstart[g + 1]; ++q) npk += P.h[chunks[order[q]].pair].npp;
                const double fl = 512.0 * nt * (npb * npk * hm_mt(L1) * hm_kt(L2) + rowt * nc * 2.0 * hm_mt(L1));
                H.hm_flops += fl;
                double* cs = H.hm_class[L1][L2][nt - 1];
                cs[0] += 1.0;
                cs[2] += fl;
                a.rows = H.d_bra.p + sb[tb];
                a.nrows = nb;
                a.chunk_ids = H.hm_chunkids.p + gstart[g];
                a.nchunks = nc;
                a.counter = H.hm_counters.p + li;
                if (prof) {
                    cudaEvent_t e0, e1;
                    CU(cudaEventCreate(&e0));
                    CU(cudaEventCreate(&e1));
                    CU(cudaEventRecord(e0, C.stream));
                    CU(hm_launch(L1, L2, nt, a, C.stream));
                    CU(cudaEventRecord(e1, C.stream));
                    timed.push_back({cs, {e0, e1}});
                } else {
                    CU(hm_launch(L1, L2, nt, a, C.aux[li % kAuxStreams]));
                }
                ++li;
            }
    }
    for (int q = 0; q < kAuxStreams; ++q) {
        CU(cudaEventRecord(C.ev_join[q], C.aux[q]));
        CU(cudaStreamWaitEvent(C.stream, C.ev_join[q], 0));
    }
    for (auto& t : timed) {
        float ms = 0.f;
        CU(cudaEventSynchronize(t.second.second));
        CU(cudaEventElapsedTime(&ms, t.second.first, t.second.second));
        t.first[1] += ms * 1e-3;
        cudaEventDestroy(t.second.first);
        cudaEventDestroy(t.second.second);
    }
}

static void run_eri(Handle& H, const std::vector<int>& bra, const std::vector<int>& ket, int mode, PairMap* rows,
                    PairMap* cols, double* out, int64_t ldo, int64_t jcount)
{
    Context& C = ctx();
    const PairTable& P = H.pt;
    const bool hm = g_hm_enabled.load() && H.hb.spher && mode != kModeDiagonal;
    // class-sorted task lists: pairs grouped by type
    std::vector<int> gb, gk;
    std::vector<int64_t> sb(kNumPairTypes + 1, 0), sk(kNumPairTypes + 1, 0);
    auto group = [&](const std::vector<int>& ids, std::vector<int>& g, std::vector<int64_t>& seg) {
        std::vector<int64_t> cnt(kNumPairTypes, 0);
        for (int id : ids) cnt[P.type[id]]++;
        seg[0] = 0;
        for (int t = 0; t < kNumPairTypes; ++t) seg[t + 1] = seg[t] + cnt[t];
        g.resize(ids.size());
        std::vector<int64_t> pos(seg.begin(), seg.end() - 1);
        for (int id : ids) g[pos[P.type[id]]++] = id;
    };
    group(bra, gb, sb);
    if (mode != kModeDiagonal) group(ket, gk, sk);
    if (hm) {
        // longest tasks first: within each pair type, pairs with more primitive
        // pairs come first, so that a launch's last tasks are its shortest
        auto by_work = [&](std::vector<int>& g, const std::vector<int64_t>& seg) {
            for (int t = 0; t < kNumPairTypes; ++t)
                std::stable_sort(g.begin() + seg[t], g.begin() + seg[t + 1],
                                 [&](int x, int y) { return P.h[x].npp > P.h[y].npp; });
        };
        by_work(gb, sb);
        by_work(gk, sk);
    }
    H.d_bra.upload(gb, C.stream);
    if (mode != kModeDiagonal) H.d_ket.upload(gk, C.stream);
    EriArgs a{};
    a.sh_xyz = H.db.xyz.p;
    a.sh_toff = H.db.toff.p;
    a.tmat = H.db.tmat.p;
    a.sh_nfunc = H.db.nfunc.p;
    a.sh_loc = H.db.loc.p;
    a.pairs = P.d.p;
    a.pp = P.pp.p;
    a.mode = mode;
    a.out = out;
    a.ldo = ldo;
    a.row_off = rows ? rows->doff.p : nullptr;
    a.row_map = rows ? rows->dmap.p : nullptr;
    a.col_off = cols ? cols->doff.p : nullptr;
    a.col_map = cols ? cols->dmap.p : nullptr;
    a.nao = H.hb.nao;
    a.jcount = jcount;
    a.kappa = H.kappa;
    a.boys = g_ctx.boys.p;
    a.err = C.err.p;
    auto sums = [&](const std::vector<int>& g, int64_t lo, int64_t hi, double& np, double& nf, double& nu) {
        np = 0.0; nf = 0.0; nu = 0.0;
        for (int64_t i = lo; i < hi; ++i) {
            const ShellPairDev& d = P.h[g[i]];
            np += (double)d.npp;
            nu += (double)d.nprim1 * d.nprim2;
            nf += (double)H.hb.nfunc[P.A[g[i]]] * H.hb.nfunc[P.B[g[i]]];
        }
    };
    for (int tb = 0; tb < kNumPairTypes; ++tb) {
        const int64_t nb = sb[tb + 1] - sb[tb];
        if (nb == 0) continue;
        double npb, nfb, nub;
        sums(gb, sb[tb], sb[tb + 1], npb, nfb, nub);
        if (mode == kModeDiagonal) {
            double np2 = 0.0, nf2 = 0.0, nu2 = 0.0;
            for (int64_t i = sb[tb]; i < sb[tb + 1]; ++i) {
                const ShellPairDev& d = P.h[gb[i]];
                const double x = (double)d.npp, y = (double)H.hb.nfunc[P.A[gb[i]]] * H.hb.nfunc[P.B[gb[i]]];
                const double u = (double)d.nprim1 * d.nprim2;
                np2 += x * x; nf2 += y * y; nu2 += u * u;
            }
            H.eri_stats[tb][tb][0] += (double)nb;
            H.eri_stats[tb][tb][1] += np2;
            H.eri_stats[tb][tb][2] += nf2;
            H.eri_stats[tb][tb][3] += nu2;
            H.eri_stats[tb][tb][4] += npb;
            H.eri_stats[tb][tb][5] += npb;
            a.bra_ids = H.d_bra.p + sb[tb];
            a.ket_ids = a.bra_ids;
            a.nbra = nb;
            a.nket = nb;
            a.swap_bk = 0;
            CU(eri_launch(tb, tb, a, C.stream));
            continue;
        }
        for (int tk = 0; tk < kNumPairTypes; ++tk) {
            const int64_t nk = sk[tk + 1] - sk[tk];
            if (nk == 0) continue;
            double npk, nfk, nuk;
            sums(gk, sk[tk], sk[tk + 1], npk, nfk, nuk);
            const int cb = std::max(tb, tk), ck = std::min(tb, tk);
            H.eri_stats[cb][ck][0] += (double)nb * nk;
            H.eri_stats[cb][ck][1] += npb * npk;
            H.eri_stats[cb][ck][2] += nfb * nfk;
            H.eri_stats[cb][ck][3] += nub * nuk;
            // primitives of the canonical bra / ket side times the quartets they enter
            H.eri_stats[cb][ck][4] += tb >= tk ? npb * (double)nk : npk * (double)nb;
            H.eri_stats[cb][ck][5] += tb >= tk ? npk * (double)nb : npb * (double)nk;
            a.bra_ids = H.d_bra.p + sb[tb];
            a.ket_ids = H.d_ket.p + sk[tk];
            a.nbra = nb;
            a.nket = nk;
            a.swap_bk = tb < tk ? 1 : 0;
            if (!hm) CU(eri_launch(std::max(tb, tk), std::min(tb, tk), a, C.stream));
        }
    }
    if (hm) run_eri_hm(H, gb, sb, gk, sk, mode, rows, cols, out, ldo, jcount);
}

// ------------------------------------------------------------------ step 1
static double accuracy_tau(int accuracy)
{
    switch (accuracy) {   // Cholesky_Gammcor.f90:398-410
    case GCI_ACCURACY_DEFAULT: return 1.0e-5;
    case GCI_ACCURACY_TIGHT: return 1.0e-6;
    case GCI_ACCURACY_LUDICROUS: return 1.0e-7;
    case GCI_ACCURACY_DEBUG: return 1.0e-10;
    default: fail(GCI_ERR_ARG, "Invalid accuracy setting");
    }
}

// C = alpha A B^T + beta C, A (m x k), B (n x k), C (m x n) column-major, on the FP64
// tensor-core GEMM (dense_fp64.cu); a_lower: A is lower triangular (Inv_L), its zero
// upper part is skipped.
static void gemm_nt(int64_t m, int64_t n, int64_t k, double alpha, const double* A, int64_t lda, const double* B,
                    int64_t ldb, double beta, double* Cm, int64_t ldc, bool a_lower = false)
{
    if (m == 0 || n == 0) return;
    DgemmArgs p{};
    p.m = m; p.n = n; p.k = k; p.alpha = alpha; p.beta = beta;
    p.a = A; p.sai = 1; p.sal = lda;
    p.b = B; p.sbl = ldb; p.sbj = 1;
    p.c = Cm; p.sci = 1; p.scj = ldc;
    p.flags = a_lower ? kDgALower : 0;
    CU(dgemm(p, 1, ctx().stream));
}

// C = alpha A B + beta C, all column-major (A m x k, B k x n), batched over `batch`
// problems at element strides sab, sbb, scb.
static void gemm_nn(int64_t m, int64_t n, int64_t k, double alpha, const double* A, int64_t lda, int64_t sab,
                    const double* B, int64_t ldb, int64_t sbb, double beta, double* Cm, int64_t ldc, int64_t scb,
                    int64_t batch, bool a_lower = false)
{
    if (m == 0 || n == 0) return;
    DgemmArgs p{};
    p.m = m; p.n = n; p.k = k; p.alpha = alpha; p.beta = beta;
    p.a = A; p.sai = 1; p.sal = lda; p.sab = sab;
    p.b = B; p.sbl = 1; p.sbj = ldb; p.sbb = sbb;
    p.c = Cm; p.sci = 1; p.scj = ldc; p.scb = scb;
    p.flags = a_lower ? kDgALower : 0;
    for (int64_t b0 = 0; b0 < batch; b0 += 65535) {
        DgemmArgs q = p;
        q.a += b0 * sab; q.b += b0 * sbb; q.c += b0 * scb;
        CU(dgemm(q, std::min<int64_t>(65535, batch - b0), ctx().stream));
    }
}

// Split-precision form of C = alpha A B^T + beta C on the int8 tensor cores
// (ozaki_gemm.cu).  A(i, l) = A[i * ars + l * als], B(j, l) = B[j * brs + l * bls],
// C column-major.  Rows of A are taken in chunks whose slice tiles fit a ~4 GB
// workspace, and K in chunks the int32 accumulators hold exactly.
static void gemm_nt_split(int64_t m, int64_t n, int64_t k, double alpha, const double* A, int64_t ars, int64_t als,
                          const double* B, int64_t brs, int64_t bls, double beta, double* Cm, int64_t ldc)
{
    if (m == 0 || n == 0) return;
    Context& C = ctx();
    if (k == 0) {
        if (beta == 1.0) return;
        fail(GCI_ERR_ARG, "split-precision GEMM with k = 0 and beta != 1");
    }
    const int64_t kmax = ozaki_max_k();
    const int64_t kc = std::min<int64_t>(k, kmax);
    const int64_t per_row = (int64_t)ozaki_workspace_bytes(128, 0, kc) / 128 + 1;
    int64_t rows = std::max<int64_t>(128, ((int64_t)4 << 30) / per_row / 128 * 128);
    rows = std::min<int64_t>(rows, (int64_t)65535 * 128);
    DVec<unsigned char> work;
    work.alloc(ozaki_workspace_bytes(std::min(rows, m), n, kc));
    for (int64_t k0 = 0; k0 < k; k0 += kc) {
        const int64_t kk = std::min(kc, k - k0);
        const double b = k0 == 0 ? beta : 1.0;
        for (int64_t r0 = 0; r0 < m; r0 += rows) {
            const int64_t mm = std::min(rows, m - r0);
            CU(ozaki_dgemm_nt(mm, n, kk, alpha, A + r0 * ars + k0 * als, ars, als, B + k0 * bls, brs, bls, b,
                              Cm + r0, ldc, work.p, C.err.p, C.stream));
        }
    }
}

// Error word of the context (set by bounded waits in the kernels that expire).
static void check_device_error(Context& C, const char* what)
{
    int e = 0;
    CU(cudaMemcpyAsync(&e, C.err.p, sizeof(int), cudaMemcpyDeviceToHost, C.stream));
    CU(cudaStreamSynchronize(C.stream));
    if (e != 0) {
        CU(cudaMemsetAsync(C.err.p, 0, sizeof(int), C.stream));
        fail(GCI_ERR_CUDA, std::string(what) + ": a bounded device wait expired");
    }
}

static void step1(Handle& H)
{
    Context& C = ctx();
    cudaStream_t s = C.stream;
    PairTable& P = H.pt;
    const HostBasis& b = H.hb;
    PhaseTimer& T = H.timer;
    const int64_t maxnorb = b.nao * (b.nao + 1) / 2;

    // ---------------- chol2_Vdiag (TwoStepCholesky_Step1.f90:202-279)
    std::vector<int> all(P.n);
    for (int64_t i = 0; i < P.n; ++i) all[i] = (int)i;
    PairMap vdm;
    vdm.reset(P.n);
    for (int64_t sp = 0; sp < P.n; ++sp) {
        const int A = P.A[sp], B = P.B[sp], Na = b.nfunc[A], Nb = b.nfunc[B];
        int* m = vdm.add((int)sp, Na * Nb);
        for (int bb = 0; bb < Nb; ++bb)
            for (int a = 0; a < Na; ++a) {
                const int64_t l = pair_local(a, bb, Na, A == B);
                m[a + Na * bb] = l < 0 ? -1 : (int)(P.vdloc[sp] + l);
            }
    }
    vdm.upload(s);
    DVec<double> dvd;
    dvd.alloc(maxnorb);
    T.start(kVdiag);
    run_eri(H, all, all, kModeDiagonal, &vdm, nullptr, dvd.p, 0);
    T.stop();
    std::vector<double> vdiag(maxnorb);
    CU(cudaMemcpyAsync(vdiag.data(), dvd.p, sizeof(double) * maxnorb, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    dvd.release();

    // ---------------- chol2_DefineBase (:282-442)
    std::vector<double> vmax(P.n);
    std::vector<int64_t> idx(P.n);
    double maxdrs = -1e300;
    for (int64_t sp = 0; sp < P.n; ++sp) {
        double m = -1e300;
        for (int i = 0; i < P.dim[sp]; ++i) m = std::max(m, vdiag[P.vdloc[sp] + i]);
        vmax[sp] = m;
        idx[sp] = sp;
        maxdrs = std::max(maxdrs, m);
    }
    if (!(maxdrs > 0.0)) fail(GCI_ERR_ARG, "Maximum diagonal Coulomb integral is nonpositive");
    const double th = std::min(H.tau, 1.0e-8);
    const double prescreen = th * th / maxdrs;
    slatec_dsort(vmax.data(), idx.data(), P.n, 2);
    int64_t k0 = 1;
    for (int64_t k = 1; k <= P.n; ++k) {
        const int64_t sp = idx[k - 1];
        double mx = -1e300;
        for (int i = 0; i < P.dim[sp]; ++i) mx = std::max(mx, vdiag[P.vdloc[sp] + i]);
        if (mx <= prescreen) k0 = k;   // the reference keeps k0 on the last discarded pair
        else break;
    }
    H.nsp = P.n - k0 + 1;
    H.bsp.resize(H.nsp);
    H.fullloc.resize(H.nsp);
    std::vector<double> D;
    {
        int64_t p = 0;
        for (int64_t k = k0, s2 = 0; k <= P.n; ++k, ++s2) {
            const int64_t sp = idx[k - 1];
            H.bsp[s2] = (int)sp;
            H.fullloc[s2] = p;
            for (int i = 0; i < P.dim[sp]; ++i) D.push_back(vdiag[P.vdloc[sp] + i]);
            p += P.dim[sp];
        }
        H.npq = p;
    }
    auto bdim = [&](int64_t s2) { return P.dim[H.bsp[s2]]; };

    // ---------------- chol2_DefineSubsets / chol2_DivideOrbPairs (:445-530)
    {
        const int64_t maxblock = 4000;   // TChol2Params%MaxBlockDim
        int64_t ns = (H.npq + maxblock - 1) / maxblock;
        if (ns < 1) ns = 1;
        H.nsubsets = ns;
        H.subsetdim.assign(ns, 0);
        H.subsetlo.assign(ns, -1);
        H.subsethi.assign(ns, -1);
        H.subloc.assign(H.nsp, 0);
        H.subidx.assign(H.nsp, 0);
        const int64_t target = (H.npq + ns - 1) / ns;
        for (int64_t k = 1; k <= ns; ++k) {
            int64_t lo;
            if (k == 1) lo = 1;
            else {
                const int64_t prev = H.subsethi[k - 2] + 1;
                lo = (prev < H.nsp && prev > 0) ? prev + 1 : 0;
            }
            int64_t dim = 0, hi = lo;
            if (lo > 0) {
                if (k < ns) {
                    int64_t berr[2] = {H.npq, H.npq}, bloc[2] = {lo, lo};
                    for (int64_t s2 = lo; s2 <= H.nsp; ++s2) {
                        H.subloc[s2 - 1] = dim;
                        H.subidx[s2 - 1] = k - 1;
                        dim += bdim(s2 - 1);
                        if (dim >= target) { bloc[1] = s2; berr[1] = dim - target; break; }
                        bloc[0] = s2; berr[0] = dim - target;
                    }
                    if (std::llabs(berr[0]) < std::llabs(berr[1])) { hi = bloc[0]; dim = berr[0] + target; }
                    else { hi = bloc[1]; dim = berr[1] + target; }
                } else {
                    hi = H.nsp;
                    for (int64_t s2 = lo; s2 <= hi; ++s2) {
                        H.subloc[s2 - 1] = dim;
                        H.subidx[s2 - 1] = k - 1;
                        dim += bdim(s2 - 1);
                    }
                }
            }
            H.subsetdim[k - 1] = dim;
            H.subsetlo[k - 1] = lo - 1;
            H.subsethi[k - 1] = hi - 1;
        }
        H.msd = *std::max_element(H.subsetdim.begin(), H.subsetdim.end());
    }

    // ---------------- chol2_Pivots (:884-1103)
    int64_t maxnchol = (int64_t)std::ceil(b.nao * 15.0);
    if (maxnchol > H.npq) maxnchol = H.npq;
    const int maxnang = H.hb.spher ? 2 * b.lmax + 1 : ncart(b.lmax);
    H.pivots.assign(H.npq, 0);
    H.pivot_order.clear();
    H.pivot_dmax.clear();

    std::vector<int64_t> cand(H.nsp), compr(H.nsp);   // candidate BASE indices; compressed loc per BASE pair
    for (int64_t k = 0; k < H.nsp; ++k) { cand[k] = k; compr[k] = H.fullloc[k]; }
    int64_t ncand = H.npq;
    DVec<double> dD, dD2;
    dD.upload(D, s);
    double dmax = *std::max_element(D.begin(), D.end());
    // vector storage over the candidates: blocks of kLBlk vectors, each ncand x kLBlk
    // column-major (ld = ncand), allocated as the vectors arrive and re-gathered block by
    // block when the candidates are compressed (the blocked V(b)%L of Step1.f90:1038-1041):
    // the peak is the vectors themselves plus one block
    constexpr int64_t kLBlk = 1024;
    std::vector<DVec<double>> Lblk;
    auto blk_cols = [&](size_t bi, int64_t nvec) { return std::min<int64_t>(kLBlk, nvec - (int64_t)bi * kLBlk); };
    const bool trace = std::getenv("GCI_TRACE_STEP1") != nullptr;
    int64_t nchol = 0;
    bool converged = false, go = maxnchol > 0;
    int64_t nmacro = 0;
    DVec<double> dM, dLB, dMbb, dDb, dLb, dpdmax, dLp, dLnew, dsegmax, dscal;
    DVec<int> dpiv, dnpiv;
    DVec<int64_t> dgidx, dsegloc, dbrow;
    DVec<int> dsegdim;
    dscal.alloc(1);
    dnpiv.alloc(1);
    std::vector<double> segmax;
    PairMap mrows, mcols;

    auto segment_max = [&](const std::vector<int64_t>& list) {
        std::vector<int64_t> loc(list.size());
        std::vector<int> dim(list.size());
        for (size_t k = 0; k < list.size(); ++k) { loc[k] = compr[list[k]]; dim[k] = bdim(list[k]); }
        dsegloc.upload(loc, s);
        dsegdim.upload(dim, s);
        dsegmax.ensure(std::max<size_t>(list.size(), 1));
        CU(launch_segmax(dD.p, dsegloc.p, dsegdim.p, (int64_t)list.size(), dsegmax.p, s));
        segmax.resize(list.size());
        if (!list.empty())
            CU(cudaMemcpyAsync(segmax.data(), dsegmax.p, sizeof(double) * list.size(), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
    };

    bool have_segmax = false;   // the candidates' maxima already read back with the last dmax
    while (go) {
        ++nmacro;
        // -------- chol2_DefineCandidates (:533-575)
        T.start(kCompress);
        if (!have_segmax) segment_max(cand);
        have_segmax = false;
        std::vector<double> sv(segmax);
        std::vector<int64_t> si(cand);
        slatec_dsort(sv.data(), si.data(), (int64_t)si.size(), -2);
        std::vector<int64_t> ncand_list;
        int64_t ncand_new = 0;
        for (size_t k = 0; k < si.size(); ++k) {
            if (sv[k] > H.tau) { ncand_list.push_back(si[k]); ncand_new += bdim(si[k]); }
            else break;
        }
        // -------- chol2_Compress (:16-97)
        {
            std::vector<int64_t> gidx(std::max<int64_t>(ncand_new, 1));
            std::vector<int64_t> newloc(ncand_list.size());
            int64_t pos = 0;
            for (size_t g = 0; g < ncand_list.size(); ++g) {
                const int64_t s2 = ncand_list[g];
                newloc[g] = pos;
                for (int i = 0; i < bdim(s2); ++i) gidx[pos + i] = compr[s2] + i;
                pos += bdim(s2);
            }
            dgidx.upload(gidx, s);
            dD2.ensure(std::max<int64_t>(ncand_new, 1));
            CU(launch_gather_rows(dD.p, ncand, dgidx.p, ncand_new, 1, dD2.p, ncand_new, s));
            std::swap(dD, dD2);
            if (ncand_new > 0) {
                for (size_t bi = 0; bi < Lblk.size(); ++bi) {
                    DVec<double> nb;
                    nb.alloc((size_t)ncand_new * kLBlk);
                    CU(launch_gather_rows(Lblk[bi].p, ncand, dgidx.p, ncand_new, blk_cols(bi, nchol), nb.p, ncand_new,
                                          s));
                    std::swap(Lblk[bi], nb);
                }
            }
            for (size_t g = 0; g < ncand_list.size(); ++g) compr[ncand_list[g]] = newloc[g];
            cand = ncand_list;
            ncand = ncand_new;
        }
        T.stop();
        int64_t maxnbatch = std::max<int64_t>((int64_t)maxnang * maxnang, 1000);
        if (maxnbatch > ncand) maxnbatch = ncand;
        const double dmin = std::max(0.01 * dmax, H.tau);
        // -------- chol2_DefineBatch (:578-625).  Its per-pair maxima of D are those just
        // sorted for the candidates (compression moves the values, it does not change
        // them), so the list is re-sorted from the host copy as the reference re-sorts it
        std::vector<double> dsv(sv.begin(), sv.begin() + (int64_t)cand.size());
        std::vector<int64_t> dsi(cand);
        slatec_dsort(dsv.data(), dsi.data(), (int64_t)dsi.size(), -2);
        std::vector<int64_t> batch, colloc;
        int64_t nbatch = 0;
        for (size_t k = 0; k < dsi.size(); ++k) {
            const int dim = bdim(dsi[k]);
            if (dsv[k] > dmin && nbatch + dim <= maxnbatch) {
                batch.push_back(dsi[k]);
                colloc.push_back(nbatch);
                nbatch += dim;
            } else break;
        }
        // -------- chol2_M (:733-856): M(ncand x nbatch)
        if (nbatch > 0 && ncand > 0) {
            mrows.reset(P.n);
            for (int64_t s2 : cand) {
                const int id = H.bsp[s2];
                const int A = P.A[id], B = P.B[id], Na = b.nfunc[A], Nb = b.nfunc[B];
                int* m = mrows.add(id, Na * Nb);
                for (int bb = 0; bb < Nb; ++bb)
                    for (int a = 0; a < Na; ++a) {
                        const int64_t l = pair_local(a, bb, Na, A == B);
                        m[a + Na * bb] = l < 0 ? -1 : (int)(compr[s2] + l);
                    }
            }
            mcols.reset(P.n);
            std::vector<int64_t> brow(nbatch);
            std::vector<int64_t> bfull(nbatch);
            for (size_t k = 0; k < batch.size(); ++k) {
                const int64_t s2 = batch[k];
                const int id = H.bsp[s2];
                const int A = P.A[id], B = P.B[id], Na = b.nfunc[A], Nb = b.nfunc[B];
                int* m = mcols.add(id, Na * Nb);
                for (int bb = 0; bb < Nb; ++bb)
                    for (int a = 0; a < Na; ++a) {
                        const int64_t l = pair_local(a, bb, Na, A == B);
                        m[a + Na * bb] = l < 0 ? -1 : (int)(colloc[k] + l);
                    }
                for (int i = 0; i < bdim(s2); ++i) {
                    brow[colloc[k] + i] = compr[s2] + i;
                    bfull[colloc[k] + i] = H.fullloc[s2] + i;
                }
            }
            mrows.upload(s);
            mcols.upload(s);
            dM.ensure((size_t)ncand * nbatch);
            std::vector<int> candids, batchids;
            for (int64_t s2 : cand) candids.push_back(H.bsp[s2]);
            for (int64_t s2 : batch) batchids.push_back(H.bsp[s2]);
            T.start(kStep1Eri);
            run_eri(H, candids, batchids, kModeProduct, &mrows, &mcols, dM.p, ncand);
            T.stop();
            // -------- chol2_SubtractR (:628-691): M -= L_cand L_batch^T
            dbrow.upload(brow, s);
            T.start(kSubtractR);
            if (nchol > 0) {
                dLB.ensure((size_t)nbatch * std::max<int64_t>(nchol, kLBlk));
                for (size_t bi = 0; bi < Lblk.size(); ++bi) {
                    const int64_t nc = blk_cols(bi, nchol);
                    double* lb = dLB.p + (size_t)bi * kLBlk * nbatch;
                    CU(launch_gather_rows(Lblk[bi].p, ncand, dbrow.p, nbatch, nc, lb, nbatch, s));
                    if (H.flags & GCI_FLAG_MIXED_STEP1)
                        gemm_nt_split(ncand, nbatch, nc, -1.0, Lblk[bi].p, 1, ncand, lb, 1, nbatch, 1.0, dM.p, ncand);
                    else
                        gemm_nt(ncand, nbatch, nc, -1.0, Lblk[bi].p, ncand, lb, nbatch, 1.0, dM.p, ncand);
                }
                H.gemm_flops[kGemmSubtractR] += 2.0 * ncand * nbatch * nchol;
            }
            T.stop();
            // -------- micro iterations (:1025-1064) on the batch block
            T.start(kPivots);
            dMbb.ensure((size_t)nbatch * nbatch);
            CU(launch_gather_rows(dM.p, ncand, dbrow.p, nbatch, nbatch, dMbb.p, nbatch, s));
            dDb.ensure(nbatch);
            CU(launch_gather_rows(dD.p, ncand, dbrow.p, nbatch, 1, dDb.p, nbatch, s));
            dLb.ensure((size_t)nbatch * nbatch);
            dpiv.ensure(nbatch);
            dpdmax.ensure(nbatch);
            CU(launch_pivot_batch(dMbb.p, (int)nbatch, dDb.p, dLb.p, dpiv.p, dpdmax.p, dnpiv.p, nchol, maxnchol, dmin, s));
            // the pivot count and the batch-length pivot lists in one read-back
            int npiv = 0;
            std::vector<int> piv(nbatch);
            std::vector<double> pdm(nbatch);
            CU(cudaMemcpyAsync(&npiv, dnpiv.p, sizeof(int), cudaMemcpyDeviceToHost, s));
            CU(cudaMemcpyAsync(piv.data(), dpiv.p, sizeof(int) * nbatch, cudaMemcpyDeviceToHost, s));
            CU(cudaMemcpyAsync(pdm.data(), dpdmax.p, sizeof(double) * nbatch, cudaMemcpyDeviceToHost, s));
            CU(cudaStreamSynchronize(s));
            piv.resize(npiv);
            pdm.resize(npiv);
            if (npiv > 0) {
                // vectors over all candidates: L_new Lp^T = M(:, piv), solved by forward
                // substitution (the column-by-column recursion of chol2_Lj,
                // Step1.f90:859-881, which stays backward stable when the batch
                // holds nearly dependent pivots; an explicit inverse does not)
                dLp.ensure((size_t)npiv * npiv);
                CU(launch_gather_pivrows(dLb.p, (int)nbatch, dpiv.p, npiv, dLp.p, s));
                dLnew.ensure((size_t)ncand * npiv);
                CU(launch_gather_cols(dM.p, ncand, dpiv.p, ncand, npiv, dLnew.p, ncand, s));
                CU(trsm_rlt(ncand, npiv, dLnew.p, ncand, dLp.p, npiv, s));
                H.gemm_flops[kGemmLnew] += (double)ncand * npiv * npiv;
                CU(launch_downdate(dD.p, dLnew.p, ncand, ncand, npiv, s));
                // append the new vectors to the blocks
                for (int64_t j = 0; j < npiv;) {
                    const int64_t col = nchol + j, bi = col / kLBlk, off = col % kLBlk;
                    if (bi == (int64_t)Lblk.size()) {
                        Lblk.emplace_back();
                        Lblk.back().alloc((size_t)ncand * kLBlk);
                    }
                    const int64_t take = std::min<int64_t>(npiv - j, kLBlk - off);
                    CU(cudaMemcpyAsync(Lblk[bi].p + off * ncand, dLnew.p + j * ncand, sizeof(double) * ncand * take,
                                       cudaMemcpyDeviceToDevice, s));
                    j += take;
                }
            }
            T.stop();
            for (int j = 0; j < npiv; ++j) {
                const int64_t full = bfull[piv[j]];
                H.pivots[full] = 1;
                H.pivot_order.push_back(full);
                H.pivot_dmax.push_back(pdm[j]);
            }
            nchol += npiv;
        }
        CU(launch_max(dD.p, ncand, dscal.p, s));
        CU(cudaMemcpyAsync(&dmax, dscal.p, sizeof(double), cudaMemcpyDeviceToHost, s));
        // the next DefineCandidates' maxima come back with dmax (segment_max synchronises)
        segment_max(cand);
        have_segmax = true;
        T.flush();
        if (ncand == 0) dmax = -1e300;
        if (trace) {
            size_t fr = 0, tot = 0;
            cudaMemGetInfo(&fr, &tot);
            std::fprintf(stderr, "step1 macro %lld: ncand %lld nbatch %lld nchol %lld dmax %.3e vectors %.2f GB free %.2f GB\n",
                         (long long)nmacro, (long long)ncand, (long long)nbatch, (long long)nchol, dmax,
                         8.0 * ncand * kLBlk * Lblk.size() / 1e9, fr / 1e9);
        }
        if (dmax <= H.tau) { converged = true; go = false; }
        if (nchol == maxnchol || nbatch == 0) go = false;
    }
    if (H.flags & GCI_FLAG_MIXED_STEP1) check_device_error(C, "split-precision M - L L^T");
    H.nvecs = nchol;
    H.nmacro = nmacro;
    H.converged = converged ? 1 : 0;
    if (nchol == maxnchol && !converged) fail(GCI_ERR_NOT_CONVERGED, "Max number of Cholesky vectors reached without convergence");
}

// ------------------------------------------------------------------ step 2
static void pq2p_ge_q(int64_t pq, int64_t n, int64_t& p, int64_t& q)
{   // chol2_pq2p_ge_q, TwoStepCholesky_Step2.f90:422-466 (1-based)
    const int64_t q_base = (pq - 1) / (n + 1) + 1;
    const int64_t v = pq - (n + 1) * (q_base - 1);
    const int64_t interval1 = n - q_base + 1;
    const int64_t in2 = v / (interval1 + 1);
    const int64_t in1 = in2 ^ 1;
    p = in1 * (q_base + v - 1) + in2 * (v - interval1 + n - q_base);
    q = in1 * q_base + in2 * interval1;
}

static void step2(Handle& H)
{
    Context& C = ctx();
    cudaStream_t s = C.stream;
    const PairTable& P = H.pt;
    const HostBasis& b = H.hb;
    PhaseTimer& T = H.timer;
    // chol2_PivotShellPairs (:469-534)
    H.psp.clear(); H.psploc.clear(); H.pspdim.clear(); H.porb.clear();
    int64_t q = 0;
    for (int64_t s2 = 0; s2 < H.nsp; ++s2) {
        const int id = H.bsp[s2];
        const int A = P.A[id], B = P.B[id], Na = b.nfunc[A];
        const int64_t p0 = H.fullloc[s2];
        const int dim = P.dim[id];
        int cnt = 0;
        for (int i = 0; i < dim; ++i) cnt += H.pivots[p0 + i];
        if (cnt == 0) continue;
        H.psp.push_back((int)s2);
        H.psploc.push_back(q);
        H.pspdim.push_back(cnt);
        for (int i = 0; i < dim; ++i) {
            if (!H.pivots[p0 + i]) continue;
            int full;
            if (A != B) full = i;
            else if (H.flags & GCI_FLAG_PIVOT_DECODE_STORAGE) {
                int bb = 0, rem = i;
                while (rem >= Na - bb) { rem -= Na - bb; ++bb; }
                full = (bb + rem) + Na * bb;
            } else {
                int64_t pa, pb;
                pq2p_ge_q(i + 1, Na, pa, pb);
                full = (int)((pa - 1) + Na * (pb - 1));
            }
            H.porb.push_back(full);
            ++q;
        }
    }
    H.npsp = (int64_t)H.psp.size();
    const int64_t N = H.nvecs;
    if (q != N) fail(GCI_ERR_STATE, "Invalid Pivots array");
    // pivot column map by pair id
    H.pivmap.reset(P.n);
    std::vector<int> pivids;
    for (int64_t k = 0; k < H.npsp; ++k) {
        const int id = H.bsp[H.psp[k]];
        pivids.push_back(id);
        int* m = H.pivmap.add(id, P.nab[id]);
        for (int r = 0; r < H.pspdim[k]; ++r) m[H.porb[H.psploc[k] + r]] = (int)(H.psploc[k] + r);
    }
    H.pivmap.upload(s);
    // chol2_Vpqrs (Step2.f90:76-187): here the full square (symmetric)
    H.invl.alloc((size_t)std::max<int64_t>(N, 1) * std::max<int64_t>(N, 1));
    if (N == 0) return;
    CU(cudaMemsetAsync(H.invl.p, 0, sizeof(double) * N * N, s));
    T.start(kVjjEri);
    run_eri(H, pivids, pivids, kModeProduct, &H.pivmap, &H.pivmap, H.invl.p, N);
    T.stop();
    // real_Cholesky + real_LowerTriangularInverse (real_linalg.f90:39-72)
    T.start(kPotrf);
    {
        // L in place of V_JJ, Inv_L into a second buffer that becomes H.invl
        DVec<double> X;
        X.alloc((size_t)N * N);
        DVec<int> info;
        info.alloc(1);
        CU(potrf_inverse(N, H.invl.p, X.p, N, info.p, s));
        int hinfo = 0;
        CU(cudaMemcpyAsync(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        if (hinfo != 0) fail(GCI_ERR_NOT_SPD, "Cholesky factorization of V_JJ failed: info=" + std::to_string(hinfo));
        std::swap(H.invl, X);
    }
    T.stop();
    H.gemm_flops[kGemmPotrf] += 2.0 * (double)N * N * N / 3.0;
    T.flush();
}

// Full-dimension vectors, one subset at a time (TwoStepCholesky.f90:378-416)
static void materialize_rkpq(Handle& H)
{
    Context& C = ctx();
    cudaStream_t s = C.stream;
    const PairTable& P = H.pt;
    const HostBasis& b = H.hb;
    const int64_t N = H.nvecs, msd = std::max<int64_t>(H.msd, 1);
    H.rkpq.alloc((size_t)std::max<int64_t>(N, 1) * msd * H.nsubsets);
    CU(cudaMemsetAsync(H.rkpq.p, 0, sizeof(double) * std::max<int64_t>(N, 1) * msd * H.nsubsets, s));
    if (N == 0) { H.have_rkpq = true; return; }
    DVec<double> W;
    W.alloc((size_t)msd * N);
    PairMap rows;
    std::vector<int> pivids;
    for (int64_t k = 0; k < H.npsp; ++k) pivids.push_back(H.bsp[H.psp[k]]);
    for (int64_t X = 0; X < H.nsubsets; ++X) {
        if (H.subsetlo[X] < 0) continue;
        rows.reset(P.n);
        std::vector<int> ids;
        for (int64_t s2 = H.subsetlo[X]; s2 <= H.subsethi[X]; ++s2) {
            const int id = H.bsp[s2];
            ids.push_back(id);
            const int A = P.A[id], B = P.B[id], Na = b.nfunc[A], Nb = b.nfunc[B];
            int* m = rows.add(id, Na * Nb);
            for (int bb = 0; bb < Nb; ++bb)
                for (int a = 0; a < Na; ++a) {
                    const int64_t l = pair_local(a, bb, Na, A == B);
                    m[a + Na * bb] = l < 0 ? -1 : (int)(H.subloc[s2] + l);
                }
        }
        rows.upload(s);
        CU(cudaMemsetAsync(W.p, 0, sizeof(double) * msd * N, s));
        H.timer.start(kFullEri);
        run_eri(H, ids, pivids, kModeProduct, &rows, &H.pivmap, W.p, msd);
        H.timer.stop();
        // real_abT: Rkpq(:,:,X) = Inv_L W^T
        H.timer.start(kInvLGemm);
        gemm_nt(N, msd, N, 1.0, H.invl.p, N, W.p, msd, 0.0, H.rkpq.p + (size_t)N * msd * X, N, true);
        H.gemm_flops[kGemmInvL] += 2.0 * N * N * (double)msd;
        H.timer.stop();
    }
    CU(cudaStreamSynchronize(s));
    H.timer.flush();
    H.have_rkpq = true;
}

// ------------------------------------------------------------------ AO -> MO
// GEMM1: W1[a][q][k] = sum_p CA[p][a] U[p][q][k]; GEMM2: out[b][a][k] = sum_q CB[q][b] W1[a][q][k]
static void mo_two_gemms(Handle& H, int precision, const double* U, int64_t kc, const double* CAd, int64_t NA,
                         const double* CBd, int64_t NB, double* W1, double* out, int64_t ldk)
{
    const int64_t nao = H.hb.nao;
    H.gemm_flops[kGemmMo] += 2.0 * (double)nao * nao * kc * NA + 2.0 * (double)kc * NB * nao * NA;
    if (precision == GCI_PREC_FP64) {
        gemm_nn(nao * kc, NA, nao, 1.0, U, nao * kc, 0, CAd, nao, 0, 0.0, W1, nao * kc, 0, 1);
        gemm_nn(kc, NB, nao, 1.0, W1, kc, nao * kc, CBd, nao, 0, 0.0, out, ldk * NA, ldk, NA);
    } else {
        // W1 (nao kc x NA) = U (rows (q,k), K = p) C_A; then per a: out_a (kc x NB) = W1_a (kc x nao) C_B
        gemm_nt_split(nao * kc, NA, nao, 1.0, U, 1, nao * kc, CAd, nao, 1, 0.0, W1, nao * kc);
        for (int64_t a = 0; a < NA; ++a)
            gemm_nt_split(kc, NB, nao, 1.0, W1 + a * nao * kc, 1, kc, CBd, nao, 1, 0.0, out + a * ldk, ldk * NA);
    }
}

static void rkab_impl(Handle& H, const double* CA, int64_t ldca, int64_t a0, int64_t a1, const double* CB_,
                      int64_t ldcb, int64_t b0, int64_t b1, int64_t max_buffer_mb, int precision, double* rkab,
                      bool device_io)
{
    Context& C = ctx();
    cudaStream_t s = C.stream;
    const PairTable& P = H.pt;
    const HostBasis& b = H.hb;
    const int64_t nao = b.nao, N = H.nvecs;
    const int64_t NA = a1 - a0 + 1, NB = b1 - b0 + 1;
    if (NA <= 0 || NB <= 0) fail(GCI_ERR_ARG, "Invalid dimension of Rkab");
    if (ldca < nao || ldcb < nao) fail(GCI_ERR_ARG, "Invalid number of atomic orbitals in CA/CB");
    if (precision != GCI_PREC_FP64 && precision != GCI_PREC_MIXED) fail(GCI_ERR_ARG, "invalid precision mode");
    if (N == 0) return;
    // MO coefficient blocks on the device
    DVec<double> dCA, dCB, dOut, U, W1;
    dCA.alloc((size_t)nao * NA);
    dCB.alloc((size_t)nao * NB);
    const cudaMemcpyKind kind = device_io ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    CU(cudaMemcpy2DAsync(dCA.p, sizeof(double) * nao, CA + ldca * (a0 - 1), sizeof(double) * ldca,
                         sizeof(double) * nao, NA, kind, s));
    CU(cudaMemcpy2DAsync(dCB.p, sizeof(double) * nao, CB_ + ldcb * (b0 - 1), sizeof(double) * ldcb,
                         sizeof(double) * nao, NB, kind, s));
    double* out_dev = rkab;
    // host output too large for the device next to Inv_L and the integral buffers: the
    // direct path stages Vab in the caller's host array and applies Inv_L column block by
    // column block from there (out of core)
    size_t free_b = 0, total_b = 0;
    CU(cudaMemGetInfo(&free_b, &total_b));
    // (GCI_RKAB_OUT_OF_CORE in the environment forces it, for tests)
    const bool ooc = !device_io && !H.have_rkpq &&
                     (8.0 * (double)N * NA * NB > 0.5 * (double)free_b || std::getenv("GCI_RKAB_OUT_OF_CORE"));
    if (!device_io && !ooc) {
        dOut.alloc((size_t)N * NA * NB);
        out_dev = dOut.p;
    }
    // chunk of the fastest index so that U + W1 fit in the buffer budget
    const double budget = (max_buffer_mb > 0 ? (double)max_buffer_mb : 8192.0) * 1024.0 * 1024.0;
    int64_t kc = (int64_t)(budget / (8.0 * (double)(nao * nao + nao * NA)));
    if (kc < 1) fail(GCI_ERR_BUFFER, "Buffer size too small for Rpq->Rab");
    kc = std::min<int64_t>(kc, N);
    U.alloc((size_t)nao * nao * kc);
    W1.alloc((size_t)nao * NA * kc);
    PhaseTimer& T = H.timer;
    T.s = s;   // this call's stream (the decomposition may have run on a batch worker's)
    if (H.have_rkpq) {
        // reference order: from the stored Rkpq (Cholesky_Gammcor.f90:143-332)
        std::vector<int64_t> pqcol;
        std::vector<int> pqao;
        for (int64_t s2 = 0; s2 < H.nsp; ++s2) {
            const int id = H.bsp[s2];
            const int A = P.A[id], B = P.B[id], Na = b.nfunc[A], Nb = b.nfunc[B];
            const int64_t X = H.subidx[s2];
            int64_t col = H.subloc[s2] + H.msd * X;
            for (int bb = 0; bb < Nb; ++bb)
                for (int a = (A == B) ? bb : 0; a < Na; ++a) {
                    pqcol.push_back(col++);
                    pqao.push_back(b.loc[A] + a);
                    pqao.push_back(b.loc[B] + bb);
                }
        }
        DVec<int64_t> dcol;
        DVec<int> dao;
        dcol.upload(pqcol, s);
        dao.upload(pqao, s);
        for (int64_t k0 = 0; k0 < N; k0 += kc) {
            const int64_t kk = std::min(kc, N - k0);
            T.start(kMoGemm);
            CU(cudaMemsetAsync(U.p, 0, sizeof(double) * nao * nao * kk, s));
            CU(launch_unpack_rkpq(H.rkpq.p, N, dcol.p, dao.p, (int64_t)pqcol.size(), k0, kk, nao, U.p, s));
            mo_two_gemms(H, precision, U.p, kk, dCA.p, NA, dCB.p, NB, W1.p, out_dev + k0, N);
            T.stop();
        }
    } else {
        // direct: V(pq, J) chunks -> Vab(J, a, b) -> Rkab = Inv_L Vab.  The Vab rows of
        // consecutive pivot chunks collect in Vc (vcap x NA NB, ld = vcap); a full Vc is
        // multiplied into the output, Rkab(k, ab) += Inv_L(k, Jv0 + l) Vc(l, ab) for k >= Jv0
        // (Inv_L is lower triangular), so no N x NA NB intermediate is held
        const int64_t nab = NA * NB;
        int64_t vcap = (int64_t)(4.0 * 1024.0 * 1024.0 * 1024.0 / (8.0 * (double)nab));
        vcap = std::min<int64_t>(std::max<int64_t>(vcap, kc), N);
        DVec<double> Vc;
        Vc.alloc((size_t)vcap * nab);
        int64_t Jv0 = 0, Jv1 = 0;   // pivot rows held in Vc
        auto flush = [&]() {
            if (Jv1 == Jv0) return;
            if (ooc) {
                // rows Jv0..Jv1 of Vab into the host array (final layout, ld = N)
                CU(cudaMemcpy2DAsync(rkab + Jv0, sizeof(double) * N, Vc.p, sizeof(double) * vcap,
                                     sizeof(double) * (Jv1 - Jv0), nab, cudaMemcpyDeviceToHost, s));
                Jv0 = Jv1;
                return;
            }
            T.start(kInvLGemm);
            gemm_nn(N - Jv0, nab, Jv1 - Jv0, 1.0, H.invl.p + Jv0 + Jv0 * N, N, 0, Vc.p, vcap, 0, Jv0 == 0 ? 0.0 : 1.0,
                    out_dev + Jv0, N, 0, 1, true);
            H.gemm_flops[kGemmInvL] += 2.0 * (double)N * (double)(Jv1 - Jv0) * (double)nab;   // dense-GEMM count
            T.stop();
            Jv0 = Jv1;
        };
        std::vector<int> baseids;
        for (int64_t s2 = 0; s2 < H.nsp; ++s2) baseids.push_back(H.bsp[s2]);
        int64_t k = 0;
        while (k < H.npsp) {
            const int64_t J0 = H.psploc[k];
            int64_t k1 = k;
            while (k1 < H.npsp && H.psploc[k1] + H.pspdim[k1] - J0 <= kc) ++k1;
            if (k1 == k) ++k1;   // one pivot pair always fits (kc >= 1 pair of at most 49 columns)
            const int64_t J1 = H.psploc[k1 - 1] + H.pspdim[k1 - 1];
            const int64_t jc = J1 - J0;
            if (jc > kc || jc > vcap) fail(GCI_ERR_BUFFER, "Buffer size too small for Rpq->Rab");
            if (J1 - Jv0 > vcap) flush();
            PairMap cm;
            cm.reset(P.n);
            std::vector<int> kids;
            for (int64_t q = k; q < k1; ++q) {
                const int id = H.bsp[H.psp[q]];
                kids.push_back(id);
                int* m = cm.add(id, P.nab[id]);
                for (int r = 0; r < H.pspdim[q]; ++r) m[H.porb[H.psploc[q] + r]] = (int)(H.psploc[q] + r - J0);
            }
            cm.upload(s);
            CU(cudaMemsetAsync(U.p, 0, sizeof(double) * nao * nao * jc, s));
            T.start(kFullEri);
            run_eri(H, baseids, kids, kModeDense, nullptr, &cm, U.p, 0, jc);
            T.stop();
            T.start(kMoGemm);
            mo_two_gemms(H, precision, U.p, jc, dCA.p, NA, dCB.p, NB, W1.p, Vc.p + (J0 - Jv0), vcap);
            T.stop();
            Jv1 = J1;
            k = k1;
        }
        flush();
        if (ooc) {
            // Rkab(:, c) = Inv_L Vab(:, c) for blocks of columns c, in place in the host array
            Vc.release();
            U.release();
            W1.release();
            CU(cudaMemGetInfo(&free_b, &total_b));
            int64_t w = (int64_t)std::min(0.4 * (double)free_b, 16.0 * 1024 * 1024 * 1024) / (16 * N);
            w = std::max<int64_t>(1, std::min(w, nab));
            DVec<double> Vin, Vout;
            Vin.alloc((size_t)N * w);
            Vout.alloc((size_t)N * w);
            T.start(kInvLGemm);
            for (int64_t c0 = 0; c0 < nab; c0 += w) {
                const int64_t cw = std::min(w, nab - c0);
                CU(cudaMemcpyAsync(Vin.p, rkab + c0 * N, sizeof(double) * N * cw, cudaMemcpyHostToDevice, s));
                gemm_nn(N, cw, N, 1.0, H.invl.p, N, 0, Vin.p, N, 0, 0.0, Vout.p, N, 0, 1, true);
                CU(cudaMemcpyAsync(rkab + c0 * N, Vout.p, sizeof(double) * N * cw, cudaMemcpyDeviceToHost, s));
            }
            H.gemm_flops[kGemmInvL] += 2.0 * (double)N * (double)N * (double)nab;
            T.stop();
        }
    }
    if (precision == GCI_PREC_MIXED) check_device_error(C, "split-precision AO->MO");
    if (!device_io && !ooc) CU(cudaMemcpyAsync(rkab, dOut.p, sizeof(double) * N * NA * NB, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    T.flush();
}

// ------------------------------------------------------------------ allocation-free ERI matrix
// The one scratch of gci_eri_pairs_noalloc.  It is static device storage of
// the library's module, so every GPU on which that module is loaded holds
// these bytes until the process exits; nothing is allocated per call.  In
// host code `g_noalloc_scratch` only names the symbol -- its device address
// on a device comes from cudaGetSymbolAddress with that device current.
constexpr size_t kNoAllocScratchBytes = (size_t)GCI_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
static std::mutex g_noalloc_mutex;
static unsigned char* g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of the scratch on device `dev` (the current device), looked
// up on the first call for that device and kept for the process.
static unsigned char* noalloc_scratch(int dev)
{
    if (dev < 0 || dev >= kNoAllocMaxDevices) fail(GCI_ERR_ARG, "device ordinal beyond the no-alloc scratch table");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            fail(GCI_ERR_CUDA, std::string("cudaGetSymbolAddress of the no-alloc scratch failed: ") +
                                   cudaGetErrorString(e));
        }
        g_noalloc_addr[dev] = (unsigned char*)p;
    }
    return g_noalloc_addr[dev];
}

// Byte offsets of the pieces placed in the scratch, each on a 256-byte boundary.
struct ScratchPlan {
    size_t end = 0;
    size_t take(size_t bytes)
    {
        const size_t at = end;
        end += (std::max<size_t>(bytes, 1) + 255) & ~(size_t)255;
        return at;
    }
};

} // namespace gci

// =================================================================== C ABI
using namespace gci;

struct gci_handle {
    Handle h;
};

// ------------------------------------------------------------------ adjoint: Coulomb energy and gradient
// Work of the last gci_coulomb_grad call: primitive quartets per (bra level, ket level).
static double g_grad_work[kGradMaxL + 1][kGradMaxL + 1];

// J = 1/2 sum D_pq (pq|rs) D_rs, dJ/dAtomCoords and (optionally) the Coulomb
// matrix, by the Hermite-vector scheme of grad_engine.cuh.  `dev` says whether
// D and jmat are device pointers; energy and grad are host pointers.
static void coulomb_grad_impl(const gci_basis* basis, double omega, const double* D, int64_t ldd, bool dev,
                              double* energy, double* grad, double* jmat, int64_t ldj)
{
    if (!D) fail(GCI_ERR_ARG, "D is NULL");
    if (!energy && !grad && !jmat) fail(GCI_ERR_ARG, "nothing requested");
    Context& C = ctx();
    CU(grad_module_init());
    Handle H;
    H.timer.s = C.stream;
    H.kappa = (omega > 0.0) ? 1.0 / (omega * omega) : 0.0;
    H.hb = make_basis(basis);
    const int64_t nao = H.hb.nao;
    if (ldd < nao) fail(GCI_ERR_ARG, "leading dimension of D too small");
    if (jmat && ldj < nao) fail(GCI_ERR_ARG, "leading dimension of jmat too small");
    setup_pairs(H);
    const PairTable& P = H.pt;
    const HostBasis& hb = H.hb;
    // primitive pairs grouped by Hermite level L = l1 + l2 of their shell pair
    constexpr int NL = kGradMaxL + 1;
    std::vector<int> lbeg(NL, 0), ln(NL, 0);
    for (int64_t sp = 0; sp < P.n; ++sp) ln[P.h[sp].l1 + P.h[sp].l2] += P.h[sp].npp;
    std::vector<int64_t> vec_off(NL, 0), hk_off(NL, 0), pot_off(NL, 0);
    int64_t ntot = 0, nvec = 0, nhk = 0, npot = 0;
    for (int L = 0; L < NL; ++L) {
        lbeg[L] = (int)ntot;
        vec_off[L] = nvec;
        hk_off[L] = nhk;
        pot_off[L] = npot;
        ntot += ln[L];
        nvec += (int64_t)ln[L] * kGradVec * grad_hb(L);
        nhk += (int64_t)ln[L] * herm_n(L);
        npot += (int64_t)ln[L] * grad_hb(L);
    }
    std::vector<int64_t> gbase(P.n);
    std::vector<int> gpair(std::max<int64_t>(ntot, 1), 0);
    {
        std::vector<int64_t> run(lbeg.begin(), lbeg.end());
        for (int64_t sp = 0; sp < P.n; ++sp) {
            const int L = P.h[sp].l1 + P.h[sp].l2;
            gbase[sp] = run[L];
            for (int i = 0; i < P.h[sp].npp; ++i) gpair[run[L] + i] = (int)sp;
            run[L] += P.h[sp].npp;
        }
    }
    DVec<int64_t> d_gbase, d_voff, d_hkoff, d_potoff;
    DVec<int> d_lbeg, d_ln, d_ppair;
    DVec<double> mP, mX, mY, mZ, vecs, hk, V, dots, Dd, Jd;
    d_gbase.upload(gbase, C.stream);
    d_voff.upload(vec_off, C.stream);
    d_hkoff.upload(hk_off, C.stream);
    d_potoff.upload(pot_off, C.stream);
    d_lbeg.upload(lbeg, C.stream);
    d_ln.upload(ln, C.stream);
    const size_t n1 = (size_t)std::max<int64_t>(ntot, 1);
    mP.alloc(n1); mX.alloc(n1); mY.alloc(n1); mZ.alloc(n1);
    d_ppair.alloc(n1);
    vecs.alloc((size_t)std::max<int64_t>(nvec, 1));
    hk.alloc((size_t)std::max<int64_t>(nhk, 1));
    V.alloc((size_t)std::max<int64_t>(npot, 1));
    dots.alloc(n1 * kGradVec);
    const double* Dp = D;
    if (!dev) {
        Dd.alloc((size_t)ldd * nao);
        CU(cudaMemcpyAsync(Dd.p, D, sizeof(double) * (size_t)ldd * nao, cudaMemcpyHostToDevice, C.stream));
        Dp = Dd.p;
    }
    const DevBasis& db = H.db;
    CU(grad_pair_vectors_launch(P.d.p, (int)P.n, d_gbase.p, d_lbeg.p, d_ln.p, d_voff.p, d_hkoff.p, db.xyz.p, db.poff.p,
                                db.exps.p, db.coefs.p, P.plist.p, db.tmat.p, db.toff.p, db.nfunc.p, db.loc.p, Dp, ldd,
                                mP.p, mX.p, mY.p, mZ.p, vecs.p, hk.p, d_ppair.p, C.stream));
    CU(cudaMemsetAsync(V.p, 0, sizeof(double) * V.n, C.stream));
    constexpr int64_t kChunk = 512;   // ket primitive pairs per warp
    for (int L1 = 0; L1 < NL; ++L1)
        for (int L2 = 0; L2 < NL; ++L2) {
            g_grad_work[L1][L2] = (double)ln[L1] * (double)ln[L2];
            if (ln[L1] == 0 || ln[L2] == 0) continue;
            GradPotArgs a{};
            a.mP = mP.p; a.mX = mX.p; a.mY = mY.p; a.mZ = mZ.p;
            a.bra_beg = lbeg[L1]; a.nbra = ln[L1];
            a.ket_beg = lbeg[L2]; a.nket = ln[L2];
            a.hk = hk.p + hk_off[L2];
            a.V = V.p + pot_off[L1];
            a.chunk = kChunk;
            a.nchunk = (ln[L2] + kChunk - 1) / kChunk;
            a.kappa = H.kappa;
            a.boys = g_ctx.boys.p;
            CU(grad_potential_launch(L1, L2, a, C.stream));
        }
    for (int L = 0; L < NL; ++L)
        CU(grad_dots_launch(lbeg[L], ln[L], grad_hb(L), vecs.p + vec_off[L], V.p + pot_off[L], dots.p, C.stream));
    if (jmat) {
        double* Jp = jmat;
        if (!dev) {
            Jd.alloc((size_t)ldj * nao);
            Jp = Jd.p;
        }
        CU(grad_coulomb_matrix_launch(P.d.p, (int)P.n, d_gbase.p, d_lbeg.p, d_potoff.p, V.p, P.pp.p, db.tmat.p,
                                      db.toff.p, db.nfunc.p, db.loc.p, Jp, ldj, C.stream));
        if (!dev)
            CU(cudaMemcpyAsync(jmat, Jd.p, sizeof(double) * (size_t)ldj * nao, cudaMemcpyDeviceToHost, C.stream));
    }
    std::vector<double> hd((size_t)n1 * kGradVec, 0.0);
    if (ntot > 0)
        CU(cudaMemcpyAsync(hd.data(), dots.p, sizeof(double) * (size_t)ntot * kGradVec, cudaMemcpyDeviceToHost,
                           C.stream));
    CU(cudaStreamSynchronize(C.stream));
    // fixed-order host reduction: deterministic energy and gradient
    double e = 0.0;
    std::vector<double> g((size_t)3 * basis->natoms, 0.0);
    for (int64_t i = 0; i < ntot; ++i) {
        const ShellPairDev& sp = P.h[gpair[i]];
        const double* d = &hd[(size_t)i * kGradVec];
        e += 0.5 * d[0];
        const int a1 = hb.atom[sp.s1], a2 = hb.atom[sp.s2];
        for (int x = 0; x < 3; ++x) {
            g[3 * a1 + x] += d[1 + x];
            g[3 * a2 + x] += d[4 + x];
        }
    }
    if (energy) *energy = e;
    if (grad) std::copy(g.begin(), g.end(), grad);
}

// chol_gammcor_Rkpq on the calling thread's context (stream).
static void rkpq_run(Handle& H, const gci_basis* basis, int accuracy, double omega, int flags)
{
    H.tau = accuracy_tau(accuracy);
    H.kappa = (omega > 0.0) ? 1.0 / (omega * omega) : 0.0;   // Cholesky_Gammcor.f90:412-421
    H.flags = flags;
    Context& C = ctx();
    H.timer.s = C.stream;
    auto t0 = std::chrono::steady_clock::now();
    H.hb = make_basis(basis);
    setup_pairs(H);
    step1(H);
    step2(H);
    if (flags & GCI_FLAG_MATERIALIZE_RKPQ) materialize_rkpq(H);
    CU(cudaStreamSynchronize(C.stream));
    H.t_rkpq = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

extern "C" {

int gci_init(void)
{
    return guarded([&] { ctx(); });
}

int gci_rkpq(const gci_basis* basis, int accuracy, double omega, int flags, gci_handle** out)
{
    if (!out) { g_last_error = "out is NULL"; return GCI_ERR_ARG; }
    *out = nullptr;
    std::unique_ptr<gci_handle> hp(new gci_handle());
    const int rc = guarded([&] { rkpq_run(hp->h, basis, accuracy, omega, flags); });
    if (rc == GCI_OK) *out = hp.release();
    else hp.reset();
    pool_trim();
    return rc;
}

int gci_rkpq_batch(int64_t nmol, const gci_basis* bases, int accuracy, double omega, int flags, int nstreams,
                   gci_handle** out)
{
    if (!bases || !out || nmol < 0) { g_last_error = "invalid argument"; return GCI_ERR_ARG; }
    for (int64_t i = 0; i < nmol; ++i) out[i] = nullptr;
    if (nmol == 0) return GCI_OK;
    // the worker contexts are shared: batches from different caller threads run one after another
    static std::mutex batch_mutex;
    std::lock_guard<std::mutex> batch_lock(batch_mutex);
    int nw = nstreams > 0 ? nstreams : 16;
    nw = (int)std::min<int64_t>(std::min(nw, 64), nmol);
    const int rc0 = guarded([&] { ensure_pool(nw); });
    if (rc0 != GCI_OK) return rc0;
    // largest molecules first (work estimate: shells^2), taken from one queue
    std::vector<int64_t> order(nmol);
    for (int64_t i = 0; i < nmol; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int64_t a, int64_t b) { return bases[a].nshells > bases[b].nshells; });
    std::vector<std::unique_ptr<gci_handle>> hs(nmol);
    std::atomic<int64_t> next{0};
    std::atomic<bool> stop{false};
    std::mutex em;
    int err_code = GCI_OK;
    int64_t err_mol = -1;
    std::string err_msg;
    auto worker = [&](int w) {
        t_cur = g_pool[w].get();
        for (;;) {
            if (stop.load()) break;
            const int64_t q = next.fetch_add(1);
            if (q >= nmol) break;
            const int64_t i = order[q];
            std::unique_ptr<gci_handle> hp(new gci_handle());
            const int rc = guarded([&] { rkpq_run(hp->h, &bases[i], accuracy, omega, flags); });
            if (rc != GCI_OK) {
                std::lock_guard<std::mutex> lock(em);
                if (err_code == GCI_OK || i < err_mol) {
                    err_code = rc;
                    err_mol = i;
                    err_msg = g_last_error;
                }
                stop.store(true);
                break;
            }
            hs[i] = std::move(hp);
        }
        t_cur = nullptr;
    };
    std::vector<std::thread> th;
    for (int w = 1; w < nw; ++w) th.emplace_back(worker, w);
    worker(0);
    for (auto& t : th) t.join();
    t_stream = g_ctx.stream;
    if (err_code != GCI_OK) {
        hs.clear();
        pool_trim();
        g_last_error = "molecule " + std::to_string(err_mol) + ": " + err_msg;
        return err_code;
    }
    for (int64_t i = 0; i < nmol; ++i) out[i] = hs[i].release();
    pool_trim();
    return GCI_OK;
}

int gci_query(const gci_handle* h, int64_t* nvecs, int64_t* max_subset_dim, int64_t* nsubsets, int64_t* norbpairs,
              int64_t* nshellpairs, int64_t* npivshellpairs)
{
    if (!h) { g_last_error = "handle is NULL"; return GCI_ERR_ARG; }
    const Handle& H = h->h;
    if (nvecs) *nvecs = H.nvecs;
    if (max_subset_dim) *max_subset_dim = H.msd;
    if (nsubsets) *nsubsets = H.nsubsets;
    if (norbpairs) *norbpairs = H.npq;
    if (nshellpairs) *nshellpairs = H.nsp;
    if (npivshellpairs) *npivshellpairs = H.npsp;
    return GCI_OK;
}

int gci_copy_rkpq(const gci_handle* h, double* dst)
{
    if (!h || !dst) { g_last_error = "NULL argument"; return GCI_ERR_ARG; }
    return guarded([&] {
        const Handle& H = h->h;
        if (!H.have_rkpq) fail(GCI_ERR_STATE, "Rkpq was not materialised (pass GCI_FLAG_MATERIALIZE_RKPQ)");
        const size_t n = (size_t)H.nvecs * H.msd * H.nsubsets;
        if (n) CU(cudaMemcpy(dst, H.rkpq.p, n * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

int gci_rkpq_columns(gci_handle* h, int64_t n, const int64_t* pq, double* out)
{
    if (!h || (n > 0 && (!pq || !out))) { g_last_error = "NULL argument"; return GCI_ERR_ARG; }
    if (n < 0) { g_last_error = "n < 0"; return GCI_ERR_ARG; }
    return guarded([&] {
        Context& C = ctx();
        cudaStream_t s = C.stream;
        Handle& H = h->h;
        const PairTable& P = H.pt;
        const HostBasis& b = H.hb;
        const int64_t N = H.nvecs;
        if (n == 0 || N == 0) return;
        // FULL orbital-pair index -> (BASE pair, index within the pair's stored block)
        std::vector<int64_t> owner(H.npq, -1);
        for (int64_t s2 = 0; s2 < H.nsp; ++s2)
            for (int i = 0; i < P.dim[H.bsp[s2]]; ++i) owner[H.fullloc[s2] + i] = s2;
        std::vector<int> first(H.npq, -1);   // output column of each requested pair (first occurrence)
        std::vector<int64_t> dup;            // (output column, its first occurrence) of repeated pairs
        std::vector<char> used(H.nsp, 0);
        for (int64_t c = 0; c < n; ++c) {
            const int64_t f = pq[c] - 1;
            if (f < 0 || f >= H.npq) fail(GCI_ERR_ARG, "orbital pair index out of range");
            if (first[f] < 0) first[f] = (int)c;
            else { dup.push_back(c); dup.push_back(first[f]); }
            used[owner[f]] = 1;
        }
        PairMap rows;
        rows.reset(P.n);
        std::vector<int> ids;
        for (int64_t s2 = 0; s2 < H.nsp; ++s2) {
            if (!used[s2]) continue;
            const int id = H.bsp[s2];
            ids.push_back(id);
            const int A = P.A[id], B = P.B[id], Na = b.nfunc[A], Nb = b.nfunc[B];
            int* m = rows.add(id, Na * Nb);
            for (int bb = 0; bb < Nb; ++bb)
                for (int a = 0; a < Na; ++a) {
                    const int64_t l = pair_local(a, bb, Na, A == B);
                    m[a + Na * bb] = l < 0 ? -1 : first[H.fullloc[s2] + l];
                }
        }
        rows.upload(s);
        std::vector<int> pivids;
        for (int64_t k = 0; k < H.npsp; ++k) pivids.push_back(H.bsp[H.psp[k]]);
        DVec<double> W, R;
        W.alloc((size_t)n * N);
        CU(cudaMemsetAsync(W.p, 0, sizeof(double) * n * N, s));
        run_eri(H, ids, pivids, kModeProduct, &rows, &H.pivmap, W.p, n);
        // R(:, pq) = Inv_L W(pq, :)^T (TwoStepCholesky.f90:410-415 for these columns)
        R.alloc((size_t)N * n);
        gemm_nt(N, n, N, 1.0, H.invl.p, N, W.p, n, 0.0, R.p, N, true);
        for (size_t d = 0; d < dup.size(); d += 2)
            CU(cudaMemcpyAsync(R.p + N * dup[d], R.p + N * dup[d + 1], sizeof(double) * N, cudaMemcpyDeviceToDevice,
                               s));
        CU(cudaMemcpyAsync(out, R.p, sizeof(double) * N * n, cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
    });
}

int gci_copy_chol2data(const gci_handle* h, int64_t* shellpairs, int64_t* shellpairloc, int64_t* shellpairdim,
                       int64_t* subsetdim, int64_t* subsetbounds, int64_t* pivots, int64_t* pivotshellpairs,
                       int64_t* pivotshellpairloc, int64_t* pivotshellpairdim, int64_t* pivotorbpairs, double* inv_l)
{
    if (!h) { g_last_error = "handle is NULL"; return GCI_ERR_ARG; }
    return guarded([&] {
        const Handle& H = h->h;
        const PairTable& P = H.pt;
        for (int64_t s2 = 0; s2 < H.nsp; ++s2) {
            const int id = H.bsp[s2];
            if (shellpairs) { shellpairs[2 * s2] = P.A[id] + 1; shellpairs[2 * s2 + 1] = P.B[id] + 1; }
            if (shellpairloc) {
                shellpairloc[3 * s2] = H.fullloc[s2] + 1;
                shellpairloc[3 * s2 + 1] = H.subloc[s2] + 1;
                shellpairloc[3 * s2 + 2] = H.subidx[s2] + 1;
            }
            if (shellpairdim) shellpairdim[s2] = P.dim[id];
        }
        for (int64_t X = 0; X < H.nsubsets; ++X) {
            if (subsetdim) subsetdim[X] = H.subsetdim[X];
            if (subsetbounds) { subsetbounds[2 * X] = H.subsetlo[X] + 1; subsetbounds[2 * X + 1] = H.subsethi[X] + 1; }
        }
        if (pivots) for (int64_t p = 0; p < H.npq; ++p) pivots[p] = H.pivots[p];
        for (int64_t k = 0; k < H.npsp; ++k) {
            if (pivotshellpairs) pivotshellpairs[k] = H.psp[k] + 1;
            if (pivotshellpairloc) pivotshellpairloc[k] = H.psploc[k] + 1;
            if (pivotshellpairdim) pivotshellpairdim[k] = H.pspdim[k];
        }
        if (pivotorbpairs) for (int64_t q = 0; q < H.nvecs; ++q) pivotorbpairs[q] = H.porb[q] + 1;
        if (inv_l && H.nvecs > 0)
            CU(cudaMemcpy(inv_l, H.invl.p, sizeof(double) * H.nvecs * H.nvecs, cudaMemcpyDeviceToHost));
    });
}

int gci_pivot_order(const gci_handle* h, int64_t* order, double* dmax)
{
    if (!h) { g_last_error = "handle is NULL"; return GCI_ERR_ARG; }
    const Handle& H = h->h;
    for (size_t j = 0; j < H.pivot_order.size(); ++j) {
        if (order) order[j] = H.pivot_order[j] + 1;
        if (dmax) dmax[j] = H.pivot_dmax[j];
    }
    return GCI_OK;
}

int gci_rkab(gci_handle* h, const double* CA, int64_t ldca, int64_t a0, int64_t a1, const double* CB,
             int64_t ldcb, int64_t b0, int64_t b1, int64_t max_buffer_mb, int precision, double* rkab)
{
    if (!h || !CA || !CB || !rkab) { g_last_error = "NULL argument"; return GCI_ERR_ARG; }
    const int rc = guarded([&] {
        auto t0 = std::chrono::steady_clock::now();
        rkab_impl(h->h, CA, ldca, a0, a1, CB, ldcb, b0, b1, max_buffer_mb, precision, rkab, false);
        h->h.t_rkab = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    });
    pool_trim();
    return rc;
}

int gci_rkab_device(gci_handle* h, const double* CA, int64_t ldca, int64_t a0, int64_t a1, const double* CB,
                    int64_t ldcb, int64_t b0, int64_t b1, int64_t max_buffer_mb, int precision, double* rkab)
{
    if (!h || !CA || !CB || !rkab) { g_last_error = "NULL argument"; return GCI_ERR_ARG; }
    const int rc = guarded([&] {
        auto t0 = std::chrono::steady_clock::now();
        rkab_impl(h->h, CA, ldca, a0, a1, CB, ldcb, b0, b1, max_buffer_mb, precision, rkab, true);
        h->h.t_rkab = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    });
    pool_trim();
    return rc;
}

int gci_stats(const gci_handle* h, double* out, int n)
{
    if (!h || !out) { g_last_error = "NULL argument"; return GCI_ERR_ARG; }
    const Handle& H = h->h;
    constexpr int ns = Handle::kNumStats;
    // [8 + ns * 100]: DMMA arithmetic issued by the Hermite-matrix kernels (flops, padding included)
    std::vector<double> v(8 + ns * kNumPairTypes * kNumPairTypes + 1, 0.0);
    v[8 + ns * kNumPairTypes * kNumPairTypes] = H.hm_flops;
    for (int i = 0; i < kNumGemm; ++i) v[i] = H.gemm_flops[i];
    for (int tb = 0; tb < kNumPairTypes; ++tb)
        for (int tk = 0; tk < kNumPairTypes; ++tk)
            for (int q = 0; q < ns; ++q) {
                v[8 + ns * (tb * kNumPairTypes + tk) + q] = H.eri_stats[tb][tk][q];
                if (q < 3) v[5 + q] += H.eri_stats[tb][tk][q];
            }
    for (int i = 0; i < n && i < (int)v.size(); ++i) out[i] = v[i];
    return GCI_OK;
}

int gci_kernel_launches(int64_t* n)
{
    if (!n) { g_last_error = "NULL argument"; return GCI_ERR_ARG; }
    *n = launches();
    return GCI_OK;
}

int gci_get_stream(void** stream)
{
    if (!stream) { g_last_error = "NULL argument"; return GCI_ERR_ARG; }
    return guarded([&] { *stream = (void*)ctx().stream; });
}

int gci_timings(const gci_handle* h, double* out, int n)
{
    if (!h || !out) { g_last_error = "NULL argument"; return GCI_ERR_ARG; }
    const Handle& H = h->h;
    double v[13];
    for (int i = 0; i < kNumPhases; ++i) v[i] = H.timer.acc[i];
    v[10] = (double)H.nmacro;
    v[11] = H.t_rkpq;
    v[12] = H.t_rkab;
    for (int i = 0; i < n && i < 13; ++i) out[i] = v[i];
    return GCI_OK;
}

void gci_free(gci_handle* h)
{
    delete h;
    pool_trim();
}

const char* gci_last_error(void) { return g_last_error.c_str(); }

int gci_boys(int m, int64_t n, const double* x, double* out)
{
    if (m < 0 || m > kBoysMaxM || n < 0 || (n > 0 && (!x || !out))) { g_last_error = "invalid argument"; return GCI_ERR_ARG; }
    return guarded([&] {
        Context& C = ctx();
        DVec<double> dx, dout;
        std::vector<double> hx(x, x + n);
        dx.upload(hx, C.stream);
        dout.alloc((size_t)std::max<int64_t>(n, 1) * (m + 1));
        CU(boys_eval_launch(m, n, dx.p, g_ctx.boys.p, dout.p, C.stream));
        if (n) CU(cudaMemcpyAsync(out, dout.p, sizeof(double) * n * (m + 1), cudaMemcpyDeviceToHost, C.stream));
        CU(cudaStreamSynchronize(C.stream));
    });
}

int gci_spher_coeffs(int L, double* U)
{
    if (L < 0 || L > 6 || !U) { g_last_error = "invalid argument"; return GCI_ERR_ARG; }
    spher_coeffs(L, U);
    return GCI_OK;
}

int gci_normalize_basis(int64_t nparams, int64_t ldprim, const int64_t* L, const int64_t* nprim, const double* exps,
                        double* coefs, double* norm_cart, int64_t ldcart, double* norm_spher, int64_t ldsph)
{
    if (nparams < 0 || !L || !nprim || !exps || !coefs) { g_last_error = "invalid argument"; return GCI_ERR_ARG; }
    for (int64_t a = 0; a < nparams; ++a) {
        if (L[a] < 0 || L[a] > 6 || nprim[a] < 1 || nprim[a] > ldprim) { g_last_error = "invalid shell"; return GCI_ERR_ARG; }
        if ((norm_cart && ldcart < ncart((int)L[a])) || (norm_spher && ldsph < 2 * L[a] + 1)) {
            g_last_error = "norm leading dimension too small";
            return GCI_ERR_ARG;
        }
    }
    normalize_basis(nparams, ldprim, L, nprim, exps, coefs, norm_cart, ldcart, norm_spher, ldsph);
    return GCI_OK;
}

int gci_eri_pairs(const gci_basis* basis, double omega, double* out, int64_t ld)
{
    if (!out) { g_last_error = "out is NULL"; return GCI_ERR_ARG; }
    return guarded([&] {
        Context& C = ctx();
        Handle H;
        H.timer.s = C.stream;
        H.kappa = (omega > 0.0) ? 1.0 / (omega * omega) : 0.0;
        H.hb = make_basis(basis);
        setup_pairs(H);
        const PairTable& P = H.pt;
        int64_t npq = 0;
        for (int64_t i = 0; i < P.n; ++i) npq += P.dim[i];
        if (ld < npq) fail(GCI_ERR_ARG, "leading dimension too small");
        PairMap m;
        m.reset(P.n);
        std::vector<int> all(P.n);
        for (int64_t sp = 0; sp < P.n; ++sp) {
            all[sp] = (int)sp;
            const int A = P.A[sp], B = P.B[sp], Na = H.hb.nfunc[A], Nb = H.hb.nfunc[B];
            int* mm = m.add((int)sp, Na * Nb);
            for (int bb = 0; bb < Nb; ++bb)
                for (int a = 0; a < Na; ++a) {
                    const int64_t l = pair_local(a, bb, Na, A == B);
                    mm[a + Na * bb] = l < 0 ? -1 : (int)(P.vdloc[sp] + l);
                }
        }
        m.upload(C.stream);
        DVec<double> d;
        d.alloc((size_t)ld * npq);
        CU(cudaMemsetAsync(d.p, 0, sizeof(double) * ld * npq, C.stream));
        run_eri(H, all, all, kModeProduct, &m, &m, d.p, ld);
        CU(cudaMemcpyAsync(out, d.p, sizeof(double) * ld * npq, cudaMemcpyDeviceToHost, C.stream));
        CU(cudaStreamSynchronize(C.stream));
    });
}

int gci_dgemm_split(int64_t m, int64_t n, int64_t k, double alpha, const double* A, int64_t lda, const double* B,
                    int64_t ldb, double beta, double* Cm, int64_t ldc)
{
    if (m < 0 || n < 0 || k < 0 || lda < std::max<int64_t>(m, 1) || ldb < std::max<int64_t>(n, 1) ||
        ldc < std::max<int64_t>(m, 1)) {
        g_last_error = "invalid GEMM dimensions";
        return GCI_ERR_ARG;
    }
    if ((m > 0 && n > 0 && k > 0) && (!A || !B || !Cm)) { g_last_error = "NULL argument"; return GCI_ERR_ARG; }
    return guarded([&] {
        Context& C = ctx();
        gemm_nt_split(m, n, k, alpha, A, 1, lda, B, 1, ldb, beta, Cm, ldc);
        check_device_error(C, "gci_dgemm_split");
        pool_trim();
    });
}

int gci_dgemm(int64_t m, int64_t n, int64_t k, double alpha, const double* A, int64_t lda, const double* B,
              int64_t ldb, double beta, double* Cm, int64_t ldc)
{
    if (m < 0 || n < 0 || k < 0 || lda < std::max<int64_t>(m, 1) || ldb < std::max<int64_t>(n, 1) ||
        ldc < std::max<int64_t>(m, 1)) {
        g_last_error = "invalid GEMM dimensions";
        return GCI_ERR_ARG;
    }
    if ((m > 0 && n > 0) && (!Cm || (k > 0 && (!A || !B)))) { g_last_error = "NULL argument"; return GCI_ERR_ARG; }
    return guarded([&] {
        Context& C = ctx();
        gemm_nt(m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc);
        CU(cudaStreamSynchronize(C.stream));
    });
}

int gci_cholesky_inverse(int64_t n, double* A, int64_t lda, double* X)
{
    if (n < 0 || lda < std::max<int64_t>(n, 1)) { g_last_error = "invalid dimensions"; return GCI_ERR_ARG; }
    if (n > 0 && (!A || !X)) { g_last_error = "NULL argument"; return GCI_ERR_ARG; }
    return guarded([&] {
        Context& C = ctx();
        DVec<int> info;
        info.alloc(1);
        CU(potrf_inverse(n, A, X, lda, info.p, C.stream));
        int hinfo = 0;
        CU(cudaMemcpyAsync(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost, C.stream));
        CU(cudaStreamSynchronize(C.stream));
        if (hinfo != 0) fail(GCI_ERR_NOT_SPD, "Cholesky factorization failed with exit code info=" + std::to_string(hinfo));
        pool_trim();
    });
}

int gci_trsm_rlt(int64_t rows, int64_t w, double* B, int64_t ldb, const double* L, int64_t ldl)
{
    if (rows < 0 || w < 0 || ldb < std::max<int64_t>(rows, 1) || ldl < std::max<int64_t>(w, 1)) {
        g_last_error = "invalid dimensions";
        return GCI_ERR_ARG;
    }
    if (rows > 0 && w > 0 && (!B || !L)) { g_last_error = "NULL argument"; return GCI_ERR_ARG; }
    return guarded([&] {
        Context& C = ctx();
        CU(trsm_rlt(rows, w, B, ldb, L, ldl, C.stream));
        CU(cudaStreamSynchronize(C.stream));
    });
}

int gci_eri_hm(int enable)
{
    const int prev = g_hm_enabled.load() ? (g_hm_profile.load() ? 2 : 1) : 0;
    if (enable >= 0) {
        g_hm_enabled.store(enable ? 1 : 0);
        g_hm_profile.store(enable == 2 ? 1 : 0);
    }
    return prev;
}

int gci_eri_hm_stats(const gci_handle* h, double* out, int n)
{
    if (!h || !out) { g_last_error = "NULL argument"; return GCI_ERR_ARG; }
    const double* v = &h->h.hm_class[0][0][0][0];
    const int tot = (kMaxPairL + 1) * (kMaxPairL + 1) * kHmMaxNT * 3;
    for (int i = 0; i < n && i < tot; ++i) out[i] = v[i];
    return GCI_OK;
}

int gci_eri_variant(int tb, int tk, int variant)
{
    const int rc = guarded([&] {
        CU(eri_module_init());
        if (variant >= 0 && eri_set_variant(tb, tk, variant) != 0)
            fail(GCI_ERR_ARG, "ERI kernel variant " + std::to_string(variant) + " is not available for class (" +
                                  std::to_string(tb) + "|" + std::to_string(tk) + ")");
        if (eri_variant(tb, tk) < 0) fail(GCI_ERR_ARG, "invalid ERI class");
    });
    return rc == GCI_OK ? eri_variant(tb, tk) : rc;
}

int gci_autotune_eri(const gci_basis* basis, int max_pairs, double* seconds)
{
    if (max_pairs <= 0) { g_last_error = "max_pairs must be positive"; return GCI_ERR_ARG; }
    return guarded([&] {
        Context& C = ctx();
        Handle H;
        H.timer.s = C.stream;
        H.hb = make_basis(basis);
        setup_pairs(H);
        const PairTable& P = H.pt;
        std::vector<std::vector<int>> by_type(kNumPairTypes);
        for (int64_t sp = 0; sp < P.n; ++sp)
            if ((int)by_type[P.type[sp]].size() < max_pairs) by_type[P.type[sp]].push_back((int)sp);
        // every slot of the sampled pairs maps into a 1024 x 1024 scratch (collisions are
        // harmless: only the launch time is measured)
        constexpr int kSide = 1024;
        PairMap m;
        m.reset(P.n);
        for (int t = 0; t < kNumPairTypes; ++t)
            for (int id : by_type[t]) {
                int* mm = m.add(id, P.nab[id]);
                for (int i = 0; i < P.nab[id]; ++i) mm[i] = (id * 37 + i) % kSide;
            }
        m.upload(C.stream);
        DVec<double> out;
        out.alloc((size_t)kSide * kSide);
        cudaEvent_t e0, e1;
        CU(cudaEventCreate(&e0));
        CU(cudaEventCreate(&e1));
        const int kVariants = eri_num_variants();
        std::vector<double> times((size_t)kNumPairTypes * kNumPairTypes * kVariants, 0.0);
        try {
            for (int tb = 0; tb < kNumPairTypes; ++tb)
                for (int tk = 0; tk <= tb; ++tk) {
                    if (by_type[tb].empty() || by_type[tk].empty()) continue;
                    const int keep = eri_variant(tb, tk);
                    int navail = 0;
                    for (int v = 0; v < kVariants; ++v)
                        if (eri_set_variant(tb, tk, v) == 0) ++navail;
                    eri_set_variant(tb, tk, keep);
                    if (navail < 2) continue;   // one kernel only: nothing to choose
                    std::vector<double> best(kVariants, -1.0);
                    for (int v = 0; v < kVariants; ++v) {
                        if (eri_set_variant(tb, tk, v) != 0) continue;
                        float ms = 0.0f, msmin = 1e30f;
                        // warm-up, timed too: a variant three times slower than the best so far is not repeated
                        CU(cudaEventRecord(e0, C.stream));
                        run_eri(H, by_type[tb], by_type[tk], kModeProduct, &m, &m, out.p, kSide);
                        CU(cudaEventRecord(e1, C.stream));
                        CU(cudaEventSynchronize(e1));
                        CU(cudaEventElapsedTime(&ms, e0, e1));
                        double bestv = -1.0;
                        for (int u = 0; u < v; ++u)
                            if (best[u] >= 0.0 && (bestv < 0.0 || best[u] < bestv)) bestv = best[u];
                        const int reps = (bestv >= 0.0 && 1e-3 * ms > 3.0 * bestv) ? 0 : 2;
                        if (reps == 0) msmin = ms;
                        for (int rep = 0; rep < reps; ++rep) {
                            CU(cudaEventRecord(e0, C.stream));
                            run_eri(H, by_type[tb], by_type[tk], kModeProduct, &m, &m, out.p, kSide);
                            CU(cudaEventRecord(e1, C.stream));
                            CU(cudaEventSynchronize(e1));
                            CU(cudaEventElapsedTime(&ms, e0, e1));
                            msmin = std::min(msmin, ms);
                        }
                        best[v] = 1e-3 * msmin;
                        times[((size_t)tb * kNumPairTypes + tk) * kVariants + v] = best[v];
                    }
                    int pick = keep;
                    for (int v = 0; v < kVariants; ++v)
                        if (best[v] >= 0.0 && (best[pick] < 0.0 || best[v] < best[pick])) pick = v;
                    eri_set_variant(tb, tk, pick);
                }
        } catch (...) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (seconds) std::copy(times.begin(), times.end(), seconds);
    });
}

int gci_eri_pairs_noalloc(const gci_basis* basis, double omega, double* out_dev, int64_t ld, void* stream)
{
    if (!out_dev) { g_last_error = "out_dev is NULL"; return GCI_ERR_ARG; }
    return guarded([&] {
        const cudaStream_t s = (cudaStream_t)stream;
        // host tables: the same basis, pair table and index maps as gci_eri_pairs
        const HostBasis hb = make_basis(basis);
        PairTable P;
        std::vector<int> plist;
        int64_t nrec = 0;
        build_pair_table(hb, P, plist, nrec);
        if (plist.empty()) plist.push_back(0);
        int64_t npq = 0;
        for (int64_t i = 0; i < P.n; ++i) npq += P.dim[i];
        if (ld < npq) fail(GCI_ERR_ARG, "leading dimension too small");
        std::vector<int64_t> moff(P.n);
        std::vector<int> mmap;
        for (int64_t sp = 0; sp < P.n; ++sp) {
            const int A = P.A[sp], B = P.B[sp], Na = hb.nfunc[A], Nb = hb.nfunc[B];
            moff[sp] = (int64_t)mmap.size();
            for (int bb = 0; bb < Nb; ++bb)
                for (int a = 0; a < Na; ++a) {
                    const int64_t l = pair_local(a, bb, Na, A == B);
                    mmap.push_back(l < 0 ? -1 : (int)(P.vdloc[sp] + l));
                }
        }
        // pair ids grouped by pair type (one kernel per class of type pair)
        std::vector<int64_t> seg(kNumPairTypes + 1, 0);
        for (int64_t sp = 0; sp < P.n; ++sp) seg[P.type[sp] + 1]++;
        for (int t = 0; t < kNumPairTypes; ++t) seg[t + 1] += seg[t];
        std::vector<int> ids(P.n);
        {
            std::vector<int64_t> pos(seg.begin(), seg.end() - 1);
            for (int64_t sp = 0; sp < P.n; ++sp) ids[pos[P.type[sp]]++] = (int)sp;
        }
        const std::vector<double> boys = boys_table(kBoysMaxM);

        // scratch layout; reject before touching the device if it does not fit
        ScratchPlan L;
        auto bytes = [](const auto& v) { return v.size() * sizeof(v[0]); };
        const size_t o_err = L.take(sizeof(int)), o_boys = L.take(bytes(boys));
        const size_t o_xyz = L.take(bytes(hb.xyz)), o_exps = L.take(bytes(hb.exps)), o_coefs = L.take(bytes(hb.coefs));
        const size_t o_tmat = L.take(bytes(hb.tmat)), o_poff = L.take(bytes(hb.poff));
        const size_t o_nfunc = L.take(bytes(hb.nfunc)), o_loc = L.take(bytes(hb.loc)), o_toff = L.take(bytes(hb.toff));
        const size_t o_pairs = L.take(bytes(P.h)), o_plist = L.take(bytes(plist));
        const size_t o_pp = L.take(sizeof(double) * (size_t)std::max<int64_t>(nrec, 1));
        const size_t o_moff = L.take(bytes(moff)), o_mmap = L.take(bytes(mmap)), o_ids = L.take(bytes(ids));
        if (L.end > kNoAllocScratchBytes)
            fail(GCI_ERR_BUFFER, "basis needs " + std::to_string(L.end) + " bytes of scratch; gci_eri_pairs_noalloc holds " +
                                     std::to_string(kNoAllocScratchBytes) + " (use gci_eri_pairs for this basis)");

        int dev = 0;
        CU(cudaGetDevice(&dev));
        unsigned char* base = noalloc_scratch(dev);
        CU(eri_module_init());
        // every piece below is rewritten on each call; the error word is cleared
        auto put = [&](size_t off, const auto& v) {
            if (!v.empty()) CU(cudaMemcpyAsync(base + off, v.data(), bytes(v), cudaMemcpyHostToDevice, s));
        };
        CU(cudaMemsetAsync(base + o_err, 0, sizeof(int), s));
        put(o_boys, boys);
        put(o_xyz, hb.xyz); put(o_exps, hb.exps); put(o_coefs, hb.coefs); put(o_tmat, hb.tmat);
        put(o_poff, hb.poff); put(o_nfunc, hb.nfunc); put(o_loc, hb.loc); put(o_toff, hb.toff);
        put(o_pairs, P.h); put(o_plist, plist); put(o_moff, moff); put(o_mmap, mmap); put(o_ids, ids);
        CU(cudaMemsetAsync(out_dev, 0, sizeof(double) * (size_t)ld * npq, s));
        auto dp = [&](size_t off) { return (double*)(base + off); };
        auto ip = [&](size_t off) { return (int*)(base + off); };
        const ShellPairDev* dpairs = (const ShellPairDev*)(base + o_pairs);
        CU(pair_records_launch(dpairs, (int)P.n, dp(o_xyz), ip(o_poff), dp(o_exps), dp(o_coefs), ip(o_plist),
                               dp(o_pp), s));
        EriArgs a{};
        a.sh_xyz = dp(o_xyz);
        a.sh_toff = ip(o_toff);
        a.tmat = dp(o_tmat);
        a.sh_nfunc = ip(o_nfunc);
        a.sh_loc = ip(o_loc);
        a.pairs = dpairs;
        a.pp = dp(o_pp);
        a.mode = kModeProduct;
        a.out = out_dev;
        a.ldo = ld;
        a.row_off = a.col_off = (const int64_t*)(base + o_moff);
        a.row_map = a.col_map = ip(o_mmap);
        a.nao = hb.nao;
        a.kappa = (omega > 0.0) ? 1.0 / (omega * omega) : 0.0;
        a.boys = dp(o_boys);
        a.err = ip(o_err);
        for (int tb = 0; tb < kNumPairTypes; ++tb)
            for (int tk = 0; tk < kNumPairTypes; ++tk) {
                const int64_t nb = seg[tb + 1] - seg[tb], nk = seg[tk + 1] - seg[tk];
                if (nb == 0 || nk == 0) continue;
                a.bra_ids = ip(o_ids) + seg[tb];
                a.ket_ids = ip(o_ids) + seg[tk];
                a.nbra = nb;
                a.nket = nk;
                a.swap_bk = tb < tk ? 1 : 0;
                CU(eri_launch(std::max(tb, tk), std::min(tb, tk), a, s));
            }
        int herr = 0;
        CU(cudaMemcpyAsync(&herr, base + o_err, sizeof(int), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        if (herr != 0) fail(GCI_ERR_CUDA, "ERI kernel reported error " + std::to_string(herr));
    });
}

int gci_coulomb_grad(const gci_basis* basis, double omega, const double* D, int64_t ldd, double* energy,
                     double* grad, double* jmat, int64_t ldj)
{
    const int rc = guarded([&] { coulomb_grad_impl(basis, omega, D, ldd, false, energy, grad, jmat, ldj); });
    pool_trim();
    return rc;
}

int gci_coulomb_grad_device(const gci_basis* basis, double omega, const double* D_dev, int64_t ldd, double* energy,
                            double* grad, double* jmat_dev, int64_t ldj)
{
    const int rc = guarded([&] { coulomb_grad_impl(basis, omega, D_dev, ldd, true, energy, grad, jmat_dev, ldj); });
    pool_trim();
    return rc;
}

int gci_coulomb_grad_work(double* out, int n)
{
    if (!out) { g_last_error = "out is NULL"; return GCI_ERR_ARG; }
    const int m = (kGradMaxL + 1) * (kGradMaxL + 1);
    for (int i = 0; i < n && i < m; ++i) out[i] = g_grad_work[i / (kGradMaxL + 1)][i % (kGradMaxL + 1)];
    return GCI_OK;
}

} // extern "C"
