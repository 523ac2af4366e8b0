// C ABI of the B200 block-tensor path (include/ltg.h).
//
// Owns device memory and streams; converts host-engine plans (ltg_host.cpp)
// into device task arrays and launches the kernels.  No exception crosses
// the boundary: every entry point returns a status code and records a
// message for ltg_last_error().
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <functional>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <queue>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/ltg.h"
#include "ltg_device.cuh"
#include "ltg_host.hpp"

namespace ltg {
int tile_cfg_count();
int tile_cfg_bm(int cfg);
int tile_cfg_bn(int cfg);
}

using namespace ltg;

namespace {

thread_local std::string g_last_error;

#define LTG_CUDA(call)                                                          \
    do {                                                                        \
        cudaError_t e_ = (call);                                                \
        if (e_ != cudaSuccess)                                                  \
            throw error(e_ == cudaErrorMemoryAllocation ? kErrOom : kErrCuda,   \
                        std::string(#call) + ": " + cudaGetErrorString(e_));    \
    } while (0)

template<class F>
int guard(F f) {
    try {
        f();
        return kOk;
    } catch (const error &e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc &) {
        g_last_error = "host allocation failed";
        return kErrOom;
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return kErrState;
    }
}

// Device buffer owned by a context.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { if (p) cudaFree(p); }
    void alloc(size_t n) {
        if (n <= bytes && p) return;
        if (p) { cudaFree(p); p = nullptr; bytes = 0; }
        if (n == 0) return;
        LTG_CUDA(cudaMalloc(&p, n));
        bytes = n;
    }
    template<class T> T *as() const { return static_cast<T *>(p); }
};

template<class T>
void upload_vec(DevBuf &d, const std::vector<T> &v, cudaStream_t s) {
    d.alloc(v.size() * sizeof(T));
    if (!v.empty()) {
        LTG_CUDA(cudaMemcpyAsync(d.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
        LTG_CUDA(cudaStreamSynchronize(s));
    }
}

}  // namespace

namespace ltg {
// Message for ltg_last_error() from entry points defined in other files.
void set_last_error(const std::string &msg) { g_last_error = msg; }
}

// Per-kernel device timing: an event pair around every launch while enabled
// (outside graph capture), summed on request.
struct KernelTiming {
    bool enabled = false;
    std::vector<cudaEvent_t> pool;
    std::vector<std::tuple<int, cudaEvent_t, cudaEvent_t>> pending;
    double ms[LTG_KERNEL_KINDS] = {};
    int64_t count[LTG_KERNEL_KINDS] = {};
};

struct ltg_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    int host_threads = 1;
    int64_t launches = 0;
    bool capturing = false;
    int nsm = 148;
    DevBuf scratch_counter;      // work-queue counters of persistent launches
    DevBuf dot_out;              // device scalar for synchronous dot products
    KernelTiming timing;
    // Bounded device waits of the tcgen05 kernels: the limit of one pipeline
    // wait, and the error word a kernel sets when a wait gave up (copied to
    // the pinned host word after every such launch and at synchronisation).
    uint64_t wait_ns = 2000000000ull;
    DevBuf wait_err;
    int32_t *wait_err_host = nullptr;
};

static std::atomic<uint64_t> g_bt_uid{1};

struct ltg_bt {
    ltg_ctx *ctx = nullptr;
    uint64_t uid = g_bt_uid++;          // never reused (cache keys)
    BlockTensorHost h;
    DevBuf arena;
    DevBuf dir_off, dir_start, dir_ext;   // block directory for fill/denominator
    bool dir_uploaded = false;
    // orbital energies of the last denominator call, kept on the device so
    // that repeated (and graph-captured) calls only launch
    std::vector<double> denom_eps;
    int32_t denom_nocc = -1;
    DevBuf denom_dev, denom_off;
};

// One launch of the plain DMMA kernel: a tile shape, its work items, and the
// tiles whose k range was cut into chunks (summed by the split reduction;
// their partial tiles at ws_off in the workspace).
struct DmmaLaunch {
    int32_t cfg = 0;
    int32_t item0 = 0, nitems = 0;
    int32_t split0 = 0, nsplits = 0;
    int64_t ws_off = 0;
};

// Grouped products of the plain FP64 path (the groups of crt_groups): the
// operand cells of every group gathered into dense panels in buf, one DMMA
// product per group into a dense result in buf, scattered into the C blocks.
struct PlainGroups {
    int32_t ngroups = 0, nunits = 0, nsunits = 0;
    double scale = 1.0;                       // ka kb kc (and d in add mode)
    DevBuf buf, pieces, units, sunits, comps, res_off, ctab, cells;
    DevBuf tasks, cblks, items, splits, ws;   // DMMA work over buf
    std::vector<DmmaLaunch> launches;
};

struct ContractExec {
    // device task arrays bound to one output tensor and coefficient set
    DevBuf tasks, cblks, items, splits, ws;
    std::unique_ptr<PlainGroups> groups;      // grouped small blocks, if any
    std::vector<DmmaLaunch> launches;
    std::vector<std::pair<int64_t, int64_t>> zero_ranges;  // assign mode: blocks not in the schedule
    std::vector<int64_t> sched_slots;
};

// A symmetrizer of two terms fused into the plain contraction's epilogue:
// the contraction's own tasks and items (no k chunks, no grouped products),
// and per scheduled C block the destinations in the symmetrized result (its
// canonical blocks that take a term of the block, each with the term's index
// mapping and sign), added atomically into the zeroed result.
struct SymExec {
    DevBuf tasks, cblks, items, drange, dests;
    std::vector<DmmaLaunch> launches;
    // small blocks as the plain path's grouped products, their results
    // scattered from the group buffer to each cell's destinations
    std::unique_ptr<PlainGroups> groups;
    DevBuf gdrange, gdcells, gdcoef;
    // modular mode: the contraction's modular exec over a host-only view of
    // its result space (kept: the exec is cached by the view's identity);
    // dests and gd* then hold the recombination's destinations
    std::unique_ptr<ltg_bt> tview;
    struct CrtExec *crt = nullptr;
    struct OzExec *oz = nullptr;               // slice modes: the slice exec over the same view
    std::vector<int64_t> nonzero_slots;      // result blocks some term reaches
    int64_t ndests = 0;
};

// Device arrays of the split-precision path for one (C tensor, coefficients,
// mode, slice count).
struct OzExec {
    int kind = 0, S = 0, chunk_kb = 1, npanels = 0, max_rows_pad = 0, nitems = 0;
    int64_t src_elems = 0, slice_bytes = 0;   // operand elements read, slice bytes written
    DevBuf panels, slices, exps, tasks, cblks, items;
    std::vector<std::pair<int64_t, int64_t>> zero_ranges;
    std::vector<int64_t> sched_slots;

};

// Device arrays of one modular split-precision contraction (crt.cu).
struct CrtExec {
    CrtParams cp{};
    int32_t npanels = 0, nitems = 0, max_rows = 0, nx = 0, ny = 0, ngroups = 0, nunits = 0;
    int64_t src_elems = 0, res_bytes = 0;   // operand elements read per pass, residue bytes written
    int64_t fused_elems = 0;                // of those, elements of row families (read once from HBM)
    int64_t exp_elems = 0;                  // elements the exponent pass reads (the others: per pass)
    int32_t sampled = 0;                    // sampled exponent bounds, checked by the residue pass
    double scale = 1.0;                     // kc (and d in add mode) times the pair coefficients' scale
    DevBuf panels, units, tasks, items, cblks, comps, ctab, cells, gidx, ex, ey, res, out;
    DevBuf cta_items;                       // products kernel: per-CTA item list offsets (ncta + 1)
    int32_t ncta = 0;
    DevBuf ext, eyt;                        // exact exponents of the sampled rows
    // row families split in one read (launch_crt_fused): families, their
    // panels and tile offsets, and the 8-row units
    DevBuf fams, famp, famt, funits;
    int32_t nfunits = 0;
    std::vector<DCrtCell> cells_host;       // the grouped products' cells, in cell order
    std::vector<std::pair<int64_t, int64_t>> zero_ranges;
    std::vector<int64_t> sched_slots;

};

struct ltg_plan {
    ltg_ctx *ctx = nullptr;
    std::map<std::tuple<uint64_t, double, double, double, int, double, int, int>,
             std::unique_ptr<OzExec>> oz;
    std::map<std::tuple<uint64_t, double, double, double, int, double, int>,
             std::unique_ptr<CrtExec>> crt;
    ltg_bt *a = nullptr, *b = nullptr;
    int forced_tile = -1;         // >= 0: every C block uses this tile shape
    int split_k = 0;              // plain DMMA k chunks per tile: 0 automatic, 1 never, 2-4 always
    bool group_products = true;   // modular mode: small C blocks grouped into larger products
    int fused_split = 0;          // modular mode: row families split in one read (kernel shape 1, 2; 0 off)
    int crt_sampled = 1;          // modular mode: sampled exponent bounds of long rows (0: exact pass)
    // caller-built task list (ltg_plan_contract2_upload): plain FP64 only,
    // coefficients absolute, no schedule of its own
    bool external = false;
    std::vector<GemmTask> ext_tasks;
    int crt_rows = 0;             // modular mode: work-item rows (128, 256; 0 default)
    int crt_stage_kb = 4;         // modular mode: k blocks per pipeline stage of the products kernel
    std::map<std::pair<int64_t, int64_t>, int> tile_override;   // autotuned (M, N) -> shape
    // the schedule (shared with the process-wide schedule cache)
    std::shared_ptr<const ContractPlan> planp = std::make_shared<const ContractPlan>();
    const ContractPlan &plan() const { return *planp; }
    // cache of device task arrays keyed by (C tensor, ka, kb, kc, add, d)
    std::map<std::tuple<uint64_t, double, double, double, int, double>,
             std::unique_ptr<ContractExec>> exec;
    // fused symmetrizers keyed by (result tensor, symmetrizer, c, ka, kb, kc)
    std::map<std::tuple<uint64_t, std::vector<int32_t>, double, double, double, double>,
             std::unique_ptr<struct SymExec>> sym;
};

struct ltg_graph {
    ltg_ctx *ctx = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

void check_ctx(ltg_ctx *c) { if (!c) throw error(kErrBadArg, "null context"); }
void check_bt(const ltg_bt *b) { if (!b) throw error(kErrBadArg, "null block tensor"); }

Perm perm_from(int n, const int32_t *p) {
    Perm r = Perm::identity(n);
    if (!p) return r;
    bool seen[kMaxOrder] = {};
    for (int i = 0; i < n; i++) {
        if (p[i] < 0 || p[i] >= n || seen[p[i]]) throw error(kErrBadArg, "invalid permutation");
        seen[p[i]] = true;
        r.p[i] = (int8_t)p[i];
    }
    return r;
}

void parse_spec(const ltg_bt_spec *s, BlockTensorHost &h) {
    if (!s) throw error(kErrBadArg, "null spec");
    const int n = s->order;
    if (n < 1 || n > kMaxOrder) throw error(kErrBadDims, "order must be 1..8");
    if (!s->dims) throw error(kErrBadArg, "null dims");
    h.bis = Bis();
    h.bis.n = n;
    int64_t pos = 0;
    for (int d = 0; d < n; d++) {
        h.bis.dims[d] = s->dims[d];
        h.bis.starts[d].clear();
        h.bis.starts[d].push_back(0);
        int ns = s->nsplit ? s->nsplit[d] : 0;
        for (int k = 0; k < ns; k++) h.bis.starts[d].push_back(s->splits[pos++]);
    }
    h.bis.finalize();
    for (int d = 0; d < n; d++) {
        h.bis.type[d] = d;
        for (int e = 0; e < d; e++)
            if (h.bis.dims[e] == h.bis.dims[d] && h.bis.starts[e] == h.bis.starts[d]) { h.bis.type[d] = h.bis.type[e]; break; }
    }
    h.sym = Symmetry();
    for (int g = 0; g < s->nperm; g++) {
        SePerm e;
        e.perm = perm_from(n, s->perm + (size_t)g * n);
        e.coeff = s->perm_coeff ? s->perm_coeff[g] : 1.0;
        if (e.coeff != 1.0 && e.coeff != -1.0) throw error(kErrSymmetry, "se_perm coefficient must be +1 or -1");
        // the permutation must map the block index space onto itself
        // (se_perm::is_valid_bis, libtensor/symmetry/se_perm.h:114-121)
        if (!h.bis.permuted(e.perm).equals(h.bis)) throw error(kErrSymmetry, "se_perm incompatible with the block index space");
        h.sym.perm.push_back(e);
    }
    (void)perm_group_closure(n, h.sym.perm);   // validates sign consistency
    if (s->has_part) {
        SePart p;
        int64_t np = 1;
        for (int d = 0; d < n; d++) {
            p.pdims[d] = s->part_pdims[d];
            if (p.pdims[d] < 1 || h.bis.bidims[d] % p.pdims[d] != 0)
                throw error(kErrSymmetry, "block count not divisible by the number of partitions");
            p.bipdims[d] = h.bis.bidims[d] / p.pdims[d];
            np *= p.pdims[d];
        }
        p.forbidden.assign(np, 0);
        for (int64_t f = 0; f < s->npart_forbidden; f++) {
            int64_t a = 0;
            for (int d = 0; d < n; d++) {
                int64_t v = s->part_forbidden[f * n + d];
                if (v < 0 || v >= p.pdims[d]) throw error(kErrBadArg, "forbidden partition index out of range");
                a = a * p.pdims[d] + v;
            }
            p.forbidden[a] = 1;
        }
        h.sym.part.push_back(p);
    }
    if (s->has_label) {
        SeLabel l;
        l.nirrep = s->label_nirrep;
        if (l.nirrep != 1 && l.nirrep != 2 && l.nirrep != 4 && l.nirrep != 8)
            throw error(kErrUnsupported, "label tables must be abelian with 1, 2, 4 or 8 irreps");
        int64_t lp = 0;
        for (int d = 0; d < n; d++) {
            l.labels[d].resize(h.bis.bidims[d]);
            for (int64_t b = 0; b < h.bis.bidims[d]; b++) {
                int v = s->labels[lp++];
                if (v >= l.nirrep) throw error(kErrBadArg, "label out of range");
                l.labels[d][b] = v < 0 ? -1 : v;
            }
        }
        // set_rule(label_set): one single-term product per intrinsic label
        // covering all dims (libtensor/symmetry/inst/se_label_impl.h:38-54)
        for (int k = 0; k < s->label_nintr; k++) {
            LabelTerm t;
            for (int d = 0; d < n; d++) t.seq[d] = 1;
            t.intr = s->label_intr[k];
            l.rule.push_back({t});
        }
        h.sym.label.push_back(l);
    }
}

void need_dev(const ltg_ctx *c) {
    if (c->device < 0) throw error(kErrState, "host-only context has no device");
}

cudaEvent_t timing_event(ltg_ctx *c) {
    if (!c->timing.pool.empty()) {
        cudaEvent_t e = c->timing.pool.back();
        c->timing.pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    LTG_CUDA(cudaEventCreate(&e));
    return e;
}

// Brackets the launches of one kernel kind with events when timing is on.
struct TimedLaunch {
    ltg_ctx *ctx;
    int kind;
    cudaEvent_t e0 = nullptr;
    TimedLaunch(ltg_ctx *c, int k) : ctx(c), kind(k) {
        if (c->timing.enabled && !c->capturing) {
            e0 = timing_event(c);
            LTG_CUDA(cudaEventRecord(e0, c->stream));
        }
    }
    void done() {
        if (!e0) return;
        cudaEvent_t e1 = timing_event(ctx);
        LTG_CUDA(cudaEventRecord(e1, ctx->stream));
        ctx->timing.pending.emplace_back(kind, e0, e1);
        e0 = nullptr;
    }
    ~TimedLaunch() { if (e0) ctx->timing.pool.push_back(e0); }
};

void collect_timing(ltg_ctx *c) {
    if (c->timing.pending.empty()) return;
    LTG_CUDA(cudaStreamSynchronize(c->stream));
    for (auto &p : c->timing.pending) {
        float ms = 0.f;
        LTG_CUDA(cudaEventElapsedTime(&ms, std::get<1>(p), std::get<2>(p)));
        c->timing.ms[std::get<0>(p)] += ms;
        c->timing.count[std::get<0>(p)]++;
        c->timing.pool.push_back(std::get<1>(p));
        c->timing.pool.push_back(std::get<2>(p));
    }
    c->timing.pending.clear();
}

void alloc_arena(ltg_bt *bt) {
    bt->h.build_directory();
    if (bt->ctx->device < 0) return;
    size_t bytes = (size_t)std::max<int64_t>(bt->h.total_elems, 1) * sizeof(double);
    bt->arena.alloc(bytes);
    LTG_CUDA(cudaMemsetAsync(bt->arena.p, 0, bytes, bt->ctx->stream));
    LTG_CUDA(cudaStreamSynchronize(bt->ctx->stream));
}

void upload_directory(ltg_bt *bt) {
    if (bt->dir_uploaded) return;
    const BlockTensorHost &h = bt->h;
    size_t nb = h.blk_abs.size();
    std::vector<int64_t> st(nb * kDevMaxOrder, 0);
    std::vector<int32_t> ex(nb * kDevMaxOrder, 1);
    int64_t bidx[kMaxOrder];
    for (size_t i = 0; i < nb; i++) {
        h.bis.unabs(h.blk_abs[i], bidx);
        for (int d = 0; d < h.bis.n; d++) {
            st[i * kDevMaxOrder + d] = h.bis.starts[d][bidx[d]];
            ex[i * kDevMaxOrder + d] = (int32_t)h.bis.block_extent(d, bidx[d]);
        }
    }
    cudaStream_t s = bt->ctx->stream;
    upload_vec(bt->dir_off, h.blk_off, s);
    upload_vec(bt->dir_start, st, s);
    upload_vec(bt->dir_ext, ex, s);
    bt->dir_uploaded = true;
}

DGenGroup gen_group(const BlockTensorHost &h) {
    DGenGroup g;
    std::memset(&g, 0, sizeof(g));
    g.order = h.bis.n;
    std::vector<SePerm> grp = perm_group_closure(h.bis.n, h.sym.perm);
    if (grp.size() > 48) throw error(kErrUnsupported, "symmetry group too large for the generator");
    g.ngroup = (int32_t)grp.size();
    for (size_t e = 0; e < grp.size(); e++) {
        for (int d = 0; d < kDevMaxOrder; d++) g.perm[e][d] = d < h.bis.n ? grp[e].perm.p[d] : 0;
        g.coeff[e] = grp[e].coeff > 0 ? 1 : -1;
    }
    for (int d = 0; d < h.bis.n; d++) g.dims[d] = h.bis.dims[d];
    return g;
}

double two_m32(double scale) { return scale * 2.3283064365386963e-10; }   // scale * 2^-32

// ------------------------------------------------------------ contraction exec

// 16-byte loads of (k, k+1) pairs need a contiguous, even-aligned k run:
// innermost k stride 1 with even extent, every other k and row stride even
// and an even base offset.
int32_t vec16_ok(int64_t off, const SubDims &rows, const SubDims &k, bool second) {
    if (k.n < 1 || off % 2 != 0) return 0;
    const int64_t *ks = second ? k.s1 : k.s0;
    if (ks[k.n - 1] != 1 || k.ext[k.n - 1] % 2 != 0) return 0;
    for (int i = 0; i < k.n - 1; i++) if (ks[i] % 2 != 0) return 0;
    for (int i = 0; i < rows.n; i++) if (rows.s0[i] % 2 != 0) return 0;
    return 1;
}

// Tile configuration per C block: the (M, N) extents pick the compiled tile
// shape with the least padded work, weighted by the relative efficiency of
// the shape (larger tiles reuse more data per load).  An autotuned table
// (ltg_autotune) overrides the weights with measured rates.
struct TileShape { int bm, bn; double eff; };
constexpr int kNumShapes = 22;
const TileShape kShapes[kNumShapes] = {
    {128, 128, 1.00}, {64, 64, 0.78}, {64, 128, 0.90}, {32, 32, 0.45},
    {80, 128, 0.97}, {96, 128, 0.98}, {48, 128, 0.85}, {112, 128, 0.99},
    {16, 128, 0.50}, {32, 128, 0.70}, {80, 192, 0.96}, {80, 192, 0.95},
    {80, 192, 0.94}, {80, 128, 0.93}, {96, 128, 0.92},
    {80, 128, 0.91}, {80, 192, 0.91}, {64, 128, 1.10},
    {80, 128, 1.00}, {80, 128, 0.95}, {64, 128, 1.05}, {128, 64, 1.05},
};
// relative rates (the m8n8k4 shapes with two CTAs per SM measured fastest:
// 64 x 128 at 30.1 TFLOP/s on a dense 6144^3 product against 26.1 for the
// best m16n8k8 shape)
double g_tile_eff[kNumShapes] = {1.00, 0.78, 0.90, 0.45, 0.97, 0.98, 0.85, 0.99, 0.50, 0.70, 0.96, 0.95,
                                 0.94, 0.93, 0.92, 0.91, 0.91, 1.10, 1.00, 0.95, 1.05, 1.05};

int pick_tile(int64_t M, int64_t N) {
    int best = 0;
    double bestc = 1e300;
    for (int c = 0; c < kNumShapes; c++) {
        const TileShape &s = kShapes[c];
        double pm = (double)((M + s.bm - 1) / s.bm) * s.bm;
        double pn = (double)((N + s.bn - 1) / s.bn) * s.bn;
        double cost = pm * pn / g_tile_eff[c];
        if (cost < bestc) { bestc = cost; best = c; }
    }
    return best;
}

// Work items of one tile shape, appended to `items` costliest first (LPT
// order for the persistent work queue).  The tail of a launch is uneven when
// its items are few and long; cutting the k range of the last items into
// equal chunks (partial tiles summed in chunk order by the split reduction,
// so results do not depend on scheduling) evens it out at the price of the
// partial tiles' traffic.  split_k 0 picks, among "no split" and the last
// 1, 2 or 4 waves' items (or all) in 2-4 chunks, the shortest launch:
// the slowest SM's work in a simulated greedy assignment (the device's
// work-queue order) at the nominal per-SM DMMA rate, plus the partial tiles'
// bytes at HBM speed; 1 never splits; 2-4 split every item in that many.
void append_launch(int cfg, std::vector<std::pair<double, DItem>> &v, const std::vector<DTask> &dt,
                   const std::vector<DCBlock> &dc, int nsm, int split_k, std::vector<DItem> &items,
                   std::vector<DSplit> &splits, int64_t &ws_elems, std::vector<DmmaLaunch> &launches) {
    if (v.empty()) return;
    std::stable_sort(v.begin(), v.end(), [](const std::pair<double, DItem> &x, const std::pair<double, DItem> &y) {
        return x.first > y.first;
    });
    const int bm = tile_cfg_bm(cfg), bn = tile_cfg_bn(cfg), bk = tile_cfg_bk(cfg);
    const size_t n = v.size();
    std::vector<int32_t> nkt(n, 0);
    for (size_t i = 0; i < n; i++) {
        const DCBlock &b = dc[v[i].second.cblk];
        for (int32_t t = b.t_begin; t < b.t_end; t++) nkt[i] += (dt[t].K + bk - 1) / bk;
    }
    const double kFmaPerSmSec = 40e12 / 2 / 148, kBytesPerSec = 6e12, kReduceLaunchSec = 4e-6;
    auto evaluate = [&](size_t first_split, int sk) {
        std::vector<double> w;
        double bytes = 0;
        for (size_t i = 0; i < n; i++) {
            const int parts = i >= first_split ? std::max(1, std::min(sk, nkt[i])) : 1;
            for (int p = 0; p < parts; p++) w.push_back(v[i].first / parts);
            if (parts > 1) bytes += (double)(2 * parts + 1) * bm * bn * 8;
        }
        std::sort(w.rbegin(), w.rend());
        std::priority_queue<double, std::vector<double>, std::greater<double>> load;
        for (int k = 0; k < std::max(1, nsm); k++) load.push(0.0);
        double mk = 0;
        for (double x : w) {
            double t = load.top() + x;
            load.pop();
            load.push(t);
            mk = std::max(mk, t);
        }
        return mk / kFmaPerSmSec + (bytes > 0 ? bytes / kBytesPerSec + kReduceLaunchSec : 0.0);
    };
    size_t first_split = n;
    int sk = 1;
    if (split_k >= 2) {
        first_split = 0;
        sk = std::min(split_k, 4);
    } else if (split_k == 0 && n > 0) {
        double best = evaluate(n, 1);
        for (int waves : {1, 2, 4, 0})
            for (int k = 2; k <= 4; k++) {
                const size_t fs = waves == 0 ? 0 : (n > (size_t)waves * nsm ? n - (size_t)waves * nsm : 0);
                const double t = evaluate(fs, k);
                if (t < best * 0.995) { best = t; first_split = fs; sk = k; }
            }
    }
    DmmaLaunch L;
    L.cfg = cfg;
    L.item0 = (int32_t)items.size();
    L.split0 = (int32_t)splits.size();
    L.ws_off = ws_elems;
    std::vector<std::pair<double, DItem>> out;
    int32_t slot = 0;
    for (size_t i = 0; i < n; i++) {
        const int parts = i >= first_split ? std::max(1, std::min(sk, nkt[i])) : 1;
        if (parts == 1) { out.push_back(v[i]); continue; }
        DSplit sp;
        sp.cblk = v[i].second.cblk; sp.m0 = v[i].second.m0; sp.n0 = v[i].second.n0;
        sp.nparts = parts; sp.slot0 = slot; sp.pad = 0;
        splits.push_back(sp);
        for (int p = 0; p < parts; p++) {
            DItem it = v[i].second;
            it.slot = slot++;
            it.kt0 = (int32_t)((int64_t)p * nkt[i] / parts);
            it.kt1 = (int32_t)((int64_t)(p + 1) * nkt[i] / parts);
            out.push_back({v[i].first / parts, it});
        }
    }
    std::stable_sort(out.begin(), out.end(), [](const std::pair<double, DItem> &x, const std::pair<double, DItem> &y) {
        return x.first > y.first;
    });
    for (auto &q : out) items.push_back(q.second);
    L.nitems = (int32_t)out.size();
    L.nsplits = (int32_t)splits.size() - L.split0;
    ws_elems += (int64_t)slot * bm * bn;
    launches.push_back(L);
}

void pack_sub(const SubDims &s, int32_t &n, int32_t *ext, int32_t *str0, int32_t *str1) {
    if (s.n > kDevMaxSub) throw error(kErrUnsupported, "too many sub-dimensions");
    for (int i = 0; i < s.n; i++)
        if (s.s0[i] < 0 || s.s0[i] > INT32_MAX || s.s1[i] < 0 || s.s1[i] > INT32_MAX)
            throw error(kErrUnsupported, "stride beyond the 32-bit range of the kernels");
    n = s.n;
    for (int i = 0; i < kDevMaxSub; i++) {
        ext[i] = i < s.n ? s.ext[i] : 1;
        if (str0) str0[i] = i < s.n ? (int32_t)s.s0[i] : 0;
        if (str1) str1[i] = i < s.n ? (int32_t)s.s1[i] : 0;
    }
}

// Caller-built tasks as the per-C-block lists of the plain path: consecutive
// tasks with the same c_off form one C block, whose C mapping is the first
// task's (C strides of m and n, fused on C strides alone).
void external_blocks(const ltg_plan *pl, double ka, double kb, double kc, std::vector<GemmTask> &tasks,
                     std::vector<CBlockTask> &cbt);

void build_plain_groups(ltg_plan *pl, const BlockTensorHost &ch, const std::vector<CBlockTask> &cbt, double kabc,
                        double post, std::vector<int32_t> &group_of, PlainGroups &pg,
                        std::vector<DCrtCell> *cells_out = nullptr);
std::vector<std::pair<int64_t, int64_t>> plain_group_shapes(ltg_plan *pl, ltg_bt *c,
                                                           const std::vector<CBlockTask> &cbt,
                                                           std::vector<int32_t> &group_of);

// Largest offset a sub-dimension group can add (strides s0, or s1).
int64_t sub_span(const SubDims &s, bool second) {
    int64_t m = 0;
    for (int i = 0; i < s.n; i++) m += (int64_t)(s.ext[i] - 1) * (second ? s.s1[i] : s.s0[i]);
    return m;
}

// Device task and C-block arrays of the plain path (post: d in add mode,
// else 1); every address a task can form must lie inside its arena (c_elems:
// the C arena's size).
void plain_task_arrays(const ltg_plan *pl, int64_t c_elems, const std::vector<GemmTask> &tasks,
                       const std::vector<CBlockTask> &cbt, double post, std::vector<DTask> &dt,
                       std::vector<DCBlock> &dc) {
    for (const GemmTask &t : tasks) {
        int64_t amax = t.a_off + sub_span(t.m, false) + sub_span(t.k, false);
        int64_t bmax = t.b_off + sub_span(t.n, false) + sub_span(t.k, true);
        int64_t cmax = t.c_off + sub_span(t.m, true) + sub_span(t.n, true);
        if (t.a_off < 0 || amax >= pl->a->h.total_elems || t.b_off < 0 || bmax >= pl->b->h.total_elems ||
            t.c_off < 0 || cmax >= c_elems)
            throw error(kErrState, "contraction task addresses outside an operand arena");
        if (t.m.total() * t.k.total() > pl->a->h.total_elems || t.n.total() * t.k.total() > pl->b->h.total_elems ||
            t.m.total() * t.n.total() > c_elems)
            throw error(kErrBadArg, "contraction task larger than its operands");
    }
    dt.assign(tasks.size(), DTask());
    for (size_t i = 0; i < tasks.size(); i++) {
        const GemmTask &t = tasks[i];
        DTask &x = dt[i];
        std::memset(&x, 0, sizeof(x));
        x.a_off = t.a_off; x.b_off = t.b_off;
        x.K = (int32_t)t.k.total();
        pack_sub(t.k, x.nk, x.kext, x.ka_str, x.kb_str);
        pack_sub(t.m, x.nm, x.mext, x.ma_str, nullptr);
        pack_sub(t.n, x.nn, x.next, x.nb_str, nullptr);
        x.vec_a = vec16_ok(t.a_off, t.m, t.k, false);
        x.vec_b = vec16_ok(t.b_off, t.n, t.k, true);
    }
    dc.assign(cbt.size(), DCBlock());
    for (size_t e = 0; e < cbt.size(); e++) {
        const CBlockTask &b = cbt[e];
        DCBlock &x = dc[e];
        std::memset(&x, 0, sizeof(x));
        x.c_off = b.c_off;
        double c0 = b.coeff0 != 0.0 ? b.coeff0 : 1.0;
        x.scale = c0 * post;
        x.M = (int32_t)b.M; x.N = (int32_t)b.N;
        pack_sub(b.cm, x.nm, x.mext, x.mc_str, nullptr);
        pack_sub(b.cn, x.nn, x.next, x.nc_str, nullptr);
        x.t_begin = b.t_begin; x.t_end = b.t_end;
        for (int32_t t = b.t_begin; t < b.t_end; t++) dt[t].coeff = tasks[t].coeff / c0;
    }
}

ContractExec *prepare_exec(ltg_plan *pl, ltg_bt *c, double ka, double kb, double kc, int add, double d) {
    auto key = std::make_tuple(c->uid, ka, kb, kc, add, add ? d : 0.0);
    auto it = pl->exec.find(key);
    if (it != pl->exec.end()) return it->second.get();
    if (pl->ctx->capturing) throw error(kErrState, "contraction not prepared before graph capture: call it once outside the capture");
    std::unique_ptr<ContractExec> ex(new ContractExec());
    std::vector<GemmTask> tasks;
    std::vector<CBlockTask> cbt;
    if (pl->external) external_blocks(pl, ka, kb, kc, tasks, cbt);
    else contract2_tasks(pl->plan(), pl->a->h, pl->b->h, c->h, ka, kb, kc, tasks, cbt);
    const double post = add ? d : 1.0;
    std::vector<DTask> dt;
    std::vector<DCBlock> dc;
    plain_task_arrays(pl, c->h.total_elems, tasks, cbt, post, dt, dc);
    // small blocks computed as grouped products
    std::vector<int32_t> group_of(cbt.size(), -1);
    if (pl->group_products && !pl->plan().coalesced && !pl->external) {
        ex->groups.reset(new PlainGroups());
        build_plain_groups(pl, c->h, cbt, ka * kb * kc, post, group_of, *ex->groups);
        if (ex->groups->ngroups == 0) ex->groups.reset();
    }
    // Work items per tile configuration, costliest first (LPT order for the
    // persistent work queue).
    std::vector<std::vector<std::pair<double, DItem>>> per_cfg(kNumShapes);
    for (size_t e = 0; e < cbt.size(); e++) {
        if (group_of[e] >= 0) continue;
        int cfg = pl->forced_tile >= 0 ? pl->forced_tile : pick_tile(cbt[e].M, cbt[e].N);
        auto ov = pl->tile_override.find({cbt[e].M, cbt[e].N});
        if (pl->forced_tile < 0 && ov != pl->tile_override.end()) cfg = ov->second;
        int bm = tile_cfg_bm(cfg), bn = tile_cfg_bn(cfg);
        for (int64_t m0 = 0; m0 < cbt[e].M; m0 += bm)
            for (int64_t n0 = 0; n0 < cbt[e].N; n0 += bn) {
                DItem it = make_item((int32_t)e, (int32_t)m0, (int32_t)n0);
                double cost = (double)bm * bn * (cbt[e].kflops + 8.0 * (cbt[e].t_end - cbt[e].t_begin));
                per_cfg[cfg].push_back({cost, it});
            }
    }
    std::vector<DItem> items;
    std::vector<DSplit> splits;
    int64_t ws_elems = 0;
    for (int cfg = 0; cfg < kNumShapes; cfg++)
        append_launch(cfg, per_cfg[cfg], dt, dc, pl->ctx->nsm, pl->split_k, items, splits, ws_elems, ex->launches);
    cudaStream_t s = pl->ctx->stream;
    upload_vec(ex->tasks, dt, s);
    upload_vec(ex->cblks, dc, s);
    upload_vec(ex->items, items, s);
    if (!splits.empty()) {
        upload_vec(ex->splits, splits, s);
        ex->ws.alloc(ws_elems * (int64_t)sizeof(double));
    }
    // blocks of C outside the schedule (zeroed in assign mode)
    std::vector<char> in_sched(c->h.blk_abs.size(), 0);
    if (pl->external) {
        std::map<int64_t, int64_t> slot_of_off;
        for (size_t sl = 0; sl < c->h.blk_off.size(); sl++) slot_of_off[c->h.blk_off[sl]] = (int64_t)sl;
        for (const CBlockTask &b : cbt) {
            auto f = slot_of_off.find(b.c_off);
            if (f == slot_of_off.end()) throw error(kErrBadArg, "a task's c_off is not the start of a block of C");
            if (in_sched[f->second]) throw error(kErrBadArg, "the tasks of one C block must be consecutive");
            if (b.c_off + sub_span(b.cm, true) + sub_span(b.cn, true) >= b.c_off + c->h.blk_size[f->second] ||
                b.M * b.N > c->h.blk_size[f->second])
                throw error(kErrBadArg, "a task's C range leaves its block");
            ex->sched_slots.push_back(f->second);
            in_sched[f->second] = 1;
        }
    }
    for (int64_t cabs : pl->external ? std::vector<int64_t>() : pl->plan().schedule) {
        int64_t sl = c->h.slot_of[cabs];
        in_sched[sl] = 1;
        ex->sched_slots.push_back(sl);
    }
    for (size_t sl = 0; sl < in_sched.size(); sl++) {
        if (in_sched[sl]) continue;
        int64_t b0 = c->h.blk_off[sl], b1 = b0 + c->h.blk_size[sl];
        if (!ex->zero_ranges.empty() && ex->zero_ranges.back().second >= b0 - 3)
            ex->zero_ranges.back().second = b1;
        else
            ex->zero_ranges.push_back({b0, b1});
    }
    ContractExec *raw = ex.get();
    pl->exec[key] = std::move(ex);
    return raw;
}

// ------------------------------------------------------------ split precision

OzExec *prepare_ozaki(ltg_plan *pl, ltg_bt *c, int mode, int S, double ka, double kb, double kc,
                      int add, double d) {
    const int kind = mode == LTG_MODE_OZAKI_INT8 ? kOzInt8 : mode == LTG_MODE_OZAKI_BF16 ? kOzBf16 : kOzE4m3;
    auto key = std::make_tuple(c->uid, ka, kb, kc, add, add ? d : 0.0, kind, S);
    auto it = pl->oz.find(key);
    if (it != pl->oz.end()) return it->second.get();
    if (pl->ctx->capturing) throw error(kErrState, "contraction not prepared before graph capture: call it once outside the capture");
    if (S < 1 || S > 8) throw error(kErrBadArg, "slice count must be 1..8");
    int beta0, beta, esz, kbe;
    int64_t maxprod;
    oz_kind_params(kind, &beta0, &beta, &esz, &kbe, &maxprod);
    std::unique_ptr<OzExec> ex(new OzExec());
    ex->kind = kind;
    ex->S = S;
    // exact accumulation: S * maxprod * Kc below 2^31 (INT32) or 2^24 (FP32)
    const int64_t lim = kind == kOzInt8 ? ((int64_t)1 << 31) - 1 : ((int64_t)1 << 24) - 1;
    int64_t kc_elems = lim / ((int64_t)S * maxprod);
    ex->chunk_kb = (int)std::max<int64_t>(1, std::min<int64_t>(kc_elems / kbe, 1 << 20));

    std::vector<GemmTask> tasks;
    std::vector<CBlockTask> cbt;
    contract2_tasks(pl->plan(), pl->a->h, pl->b->h, c->h, ka, kb, kc, tasks, cbt);
    // panels, de-duplicated by (operand, block, row mapping, k mapping)
    std::map<std::vector<int64_t>, int32_t> pidx;
    std::vector<DPanel> panels;
    int64_t slice_bytes = 0;
    int32_t exp_rows = 0;
    auto panel_of = [&](int src, int64_t off, const SubDims &rows, const SubDims &k, bool kb_second) {
        std::vector<int64_t> key = {src, off, rows.n, k.n};
        for (int i = 0; i < rows.n; i++) { key.push_back(rows.ext[i]); key.push_back(rows.s0[i]); }
        for (int i = 0; i < k.n; i++) { key.push_back(k.ext[i]); key.push_back(kb_second ? k.s1[i] : k.s0[i]); }
        auto f = pidx.find(key);
        if (f != pidx.end()) return f->second;
        DPanel p;
        std::memset(&p, 0, sizeof(p));
        p.src = src;
        p.src_off = off;
        p.rows = (int32_t)rows.total();
        p.K = (int32_t)k.total();
        p.rows_pad = (p.rows + 127) / 128 * 128;
        p.K_pad = (p.K + 31) / 32 * 32;      // whole 32-element split steps (a multiple of kbe)
        pack_sub(rows, p.nr, p.rext, p.rstr, nullptr);
        SubDims kk = k;
        if (kb_second) for (int i = 0; i < kk.n; i++) kk.s0[i] = kk.s1[i];
        pack_sub(kk, p.nk, p.kext, p.kstr, nullptr);
        p.slice_off = slice_bytes;
        slice_bytes += ((int64_t)S * p.rows_pad * p.K_pad * esz + 1023) / 1024 * 1024;
        p.exp_off = exp_rows;
        exp_rows += p.rows_pad;
        int32_t id = (int32_t)panels.size();
        panels.push_back(p);
        pidx[key] = id;
        return id;
    };
    std::vector<DOzTask> dt(tasks.size());
    for (size_t i = 0; i < tasks.size(); i++) {
        const GemmTask &t = tasks[i];
        dt[i].pa = panel_of(0, t.a_off, t.m, t.k, false);
        dt[i].pb = panel_of(1, t.b_off, t.n, t.k, true);
        if (panels[dt[i].pa].K_pad != panels[dt[i].pb].K_pad) throw error(kErrState, "panel k extents differ");
    }
    std::vector<DCBlock> dc(cbt.size());
    double post = add ? d : 1.0;
    for (size_t e = 0; e < cbt.size(); e++) {
        const CBlockTask &b = cbt[e];
        DCBlock &x = dc[e];
        std::memset(&x, 0, sizeof(x));
        x.c_off = b.c_off;
        double c0 = b.coeff0 != 0.0 ? b.coeff0 : 1.0;
        x.scale = c0 * post;
        x.M = (int32_t)b.M; x.N = (int32_t)b.N;
        pack_sub(b.cm, x.nm, x.mext, x.mc_str, nullptr);
        pack_sub(b.cn, x.nn, x.next, x.nc_str, nullptr);
        x.t_begin = b.t_begin; x.t_end = b.t_end;
        for (int32_t t = b.t_begin; t < b.t_end; t++) dt[t].coeff = tasks[t].coeff / c0;
    }
    // (C block, 128 x 64 tile) work items, costliest first, dealt round-robin
    std::vector<std::pair<double, DItem>> iv;
    for (size_t e = 0; e < cbt.size(); e++)
        for (int64_t m0 = 0; m0 < cbt[e].M; m0 += 128)
            for (int64_t n0 = 0; n0 < cbt[e].N; n0 += 64) {
                DItem it = make_item((int32_t)e, (int32_t)m0, (int32_t)n0);
                iv.push_back({cbt[e].kflops + 64.0 * (cbt[e].t_end - cbt[e].t_begin), it});
            }
    std::stable_sort(iv.begin(), iv.end(), [](const std::pair<double, DItem> &x, const std::pair<double, DItem> &y) { return x.first > y.first; });
    std::vector<DItem> items;
    for (auto &p : iv) items.push_back(p.second);
    for (const DPanel &p : panels) {
        ex->max_rows_pad = std::max(ex->max_rows_pad, p.rows_pad);
        ex->src_elems += (int64_t)p.rows * p.K;
        ex->slice_bytes += (int64_t)S * p.rows_pad * p.K_pad * esz;
    }

    cudaStream_t s = pl->ctx->stream;
    ex->npanels = (int)panels.size();
    ex->nitems = (int)items.size();
    ex->slices.alloc(std::max<int64_t>(slice_bytes, 1024));
    ex->exps.alloc(std::max<int32_t>(exp_rows, 1) * sizeof(int32_t));
    upload_vec(ex->panels, panels, s);
    upload_vec(ex->tasks, dt, s);
    upload_vec(ex->cblks, dc, s);
    upload_vec(ex->items, items, s);
    // blocks of C outside the schedule (zeroed in assign mode)
    std::vector<char> in_sched(c->h.blk_abs.size(), 0);
    for (int64_t cabs : pl->plan().schedule) {
        int64_t sl = c->h.slot_of[cabs];
        in_sched[sl] = 1;
        ex->sched_slots.push_back(sl);
    }
    for (size_t sl = 0; sl < in_sched.size(); sl++) {
        if (in_sched[sl]) continue;
        int64_t b0 = c->h.blk_off[sl], b1 = b0 + c->h.blk_size[sl];
        if (!ex->zero_ranges.empty() && ex->zero_ranges.back().second >= b0 - 3) ex->zero_ranges.back().second = b1;
        else ex->zero_ranges.push_back({b0, b1});
    }
    LTG_CUDA(cudaStreamSynchronize(s));
    OzExec *raw = ex.get();
    pl->oz[key] = std::move(ex);
    return raw;
}

// ------------------------------------------------------------ modular split precision

// Pairwise coprime moduli <= 256, largest first (residues fit INT8).
const int32_t kCrtModuli[kCrtMaxModuli] = {256, 255, 253, 251, 247, 241, 239, 233,
                                           229, 227, 223, 217, 211, 199, 197, 193};

int32_t mod_inverse(int64_t a, int64_t m) {
    int64_t t = 0, nt = 1, r = m, nr = ((a % m) + m) % m;
    while (nr != 0) {
        int64_t q = r / nr, tmp;
        tmp = t - q * nt; t = nt; nt = tmp;
        tmp = r - q * nr; r = nr; nr = tmp;
    }
    if (r != 1) throw error(kErrState, "moduli not coprime");
    return (int32_t)(t < 0 ? t + m : t);
}

CrtParams crt_params(int L, int P, bool swap) {
    CrtParams cp{};
    cp.L = L; cp.P = P; cp.swap = swap ? 1 : 0;
    for (int i = 0; i < L; i++) {
        const int32_t m = kCrtModuli[i];
        cp.m[i] = m;
        cp.minv_d[i] = 1.0 / (double)m;
        for (int j = 0; j < i; j++) (void)mod_inverse(kCrtModuli[j], m);   // pairwise coprime
    }
    return cp;
}

// Tile width of the MMA N operand for a panel of `rows` rows: tiles of at
// most 256 rows, balanced, in multiples of 16.
int32_t crt_tile_width(int64_t rows) {
    const int64_t nt = (rows + 255) / 256;
    const int64_t w = (rows + nt - 1) / nt;
    return (int32_t)std::min<int64_t>(256, (w + 15) / 16 * 16);
}

// Global index of every row (or column) of a C block: the C element's dense
// coordinates over the dims of that side, linearised with full extents.  The
// exponent tables are indexed by it, so that all panels feeding one row of C
// share its scaling.
struct CrtSideMap {
    std::vector<int> dims;       // C dims of this side
    std::vector<int64_t> gstr;   // strides of the linearised index
    int64_t size = 1;
};

void crt_global_index(const BlockTensorHost &ch, const CrtSideMap &sm, int64_t c_off, const SubDims &sub,
                      std::map<int64_t, int64_t> &slot_of_off, std::vector<int32_t> &out) {
    auto f = slot_of_off.find(c_off);
    if (f == slot_of_off.end()) throw error(kErrState, "C block offset without a slot");
    const int n = ch.bis.n;
    int64_t bidx[kMaxOrder], bext[kMaxOrder], bstr[kMaxOrder];
    ch.bis.unabs(ch.blk_abs[f->second], bidx);
    ch.bis.block_dims(bidx, bext);
    int64_t acc = 1;
    for (int d = n - 1; d >= 0; d--) { bstr[d] = acc; acc *= bext[d]; }
    const int64_t total = sub.total();
    out.resize(total);
    for (int64_t r = 0; r < total; r++) {
        int64_t off = 0, q = r;
        for (int i = sub.n - 1; i >= 0; i--) {
            off += (q % sub.ext[i]) * sub.s1[i];
            q /= sub.ext[i];
        }
        int64_t g = 0;
        for (size_t k = 0; k < sm.dims.size(); k++) {
            const int d = sm.dims[k];
            const int64_t local = (off / bstr[d]) % bext[d];
            g += (ch.bis.starts[d][bidx[d]] + local) * sm.gstr[k];
        }
        out[r] = (int32_t)g;
    }
}

// ---- grouped modular products
//
// Without coalescing, the pair list of a C block (R, S) (R: its block
// indices on the C dims taken from A, S: on those taken from B) holds every
// contracted block index K whose A block (R, K) and B block (K, S) are both
// non-zero (gen_bto_contract2_clst_builder).  So for any set of row blocks and
// column blocks, the product of [A(R, K)] (rows R, columns K over the union of
// the contracted blocks, zero where no pair uses the cell) and [B(K, S)] holds,
// in cell (R, S), exactly the sum over the pairs of C block (R, S).  The
// schedule links row and column blocks; each connected set of them becomes one
// grouped product when its grid is dense enough.

// One operand cell: the canonical block read with the pair's orbit transform,
// rows = the C dims of its side in C order, k = the contracted dims in the
// order of A's dims (the same for the A and the B cell of one K).
struct CrtCell {
    int64_t off = 0;
    int32_t coef = 1;
    SubDims rows, k;              // s0: stride in the operand's canonical block
};

struct CrtGroupHost {
    std::vector<int64_t> rkey, skey, kkey;     // row / column / contracted block keys, ascending
    std::vector<int64_t> rn, sn, kn;           // their extents
    std::vector<int32_t> rce, sce;             // a C block (cbt index) holding each row / column block
    std::vector<int32_t> cell;                 // rkey.size() x skey.size(): cbt index or -1
    std::map<std::pair<int32_t, int32_t>, CrtCell> ac, bc;   // (R, K) -> A cell, (K, S) -> B cell
};

// Strides fused where contiguous (same linear order), unit extents dropped.
SubDims fuse_single(int n, const int64_t *ext, const int64_t *str) {
    SubDims r;
    for (int i = 0; i < n; i++) {
        if (ext[i] == 1) continue;
        if (r.n > 0 && r.s0[r.n - 1] == str[i] * ext[i]) {
            r.ext[r.n - 1] *= (int32_t)ext[i];
            r.s0[r.n - 1] = str[i];
            continue;
        }
        if (r.n == kMaxSub) throw error(kErrUnsupported, "too many sub-dimensions");
        r.ext[r.n] = (int32_t)ext[i]; r.s0[r.n] = str[i]; r.n++;
    }
    return r;
}

int32_t round4(int64_t x) { return (int32_t)((x + 3) / 4 * 4); }

// C dims of each side: connected to A (rows) or to B (columns), and the
// strides of the linearised global index of each side.
void crt_side_maps(const Contraction &ct, const BlockTensorHost &ch, CrtSideMap *sm) {
    for (int i = 0; i < ct.NC(); i++) sm[ct.conn[i] < ct.NC() + ct.NA() ? 0 : 1].dims.push_back(i);
    for (int s = 0; s < 2; s++) {
        sm[s].gstr.resize(sm[s].dims.size());
        for (int k = (int)sm[s].dims.size() - 1; k >= 0; k--) {
            sm[s].gstr[k] = sm[s].size;
            sm[s].size *= ch.bis.dims[sm[s].dims[k]];
        }
        if (sm[s].size > ((int64_t)1 << 27)) throw error(kErrUnsupported, "C side too large for the modular scaling tables");
    }
}

void crt_groups(const ltg_plan *pl, const BlockTensorHost &ch, const CrtSideMap *sm,
                const std::vector<CBlockTask> &cbt, std::vector<CrtGroupHost> &groups,
                std::vector<int32_t> &group_of) {
    const ContractPlan &P = pl->plan();
    const Contraction &c0 = P.contr;
    const BlockTensorHost &ah = pl->a->h, &bh = pl->b->h;
    const int NC = c0.NC(), NA = c0.NA(), NB = c0.NB();
    const size_t ne = cbt.size();
    group_of.assign(ne, -1);
    if (ne < 2) return;
    if (sm[0].dims.size() > (size_t)kCrtSideDims || sm[1].dims.size() > (size_t)kCrtSideDims) return;
    // contracted dims of A in A order (the k order of every cell)
    std::vector<int> kdims;
    for (int i = 0; i < NA; i++) if (c0.conn[NC + i] >= NC + NA) kdims.push_back(i);

    int64_t ic[kMaxOrder];
    auto side_key = [&](int s) {
        int64_t k = 0;
        for (int d : sm[s].dims) k = k * ch.bis.bidims[d] + ic[d];
        return k;
    };
    std::map<int64_t, int32_t> rid, sid;
    std::vector<int32_t> er(ne), es(ne);
    for (size_t e = 0; e < ne; e++) {
        ch.bis.unabs(P.schedule[e], ic);
        er[e] = rid.emplace(side_key(0), (int32_t)rid.size()).first->second;
        es[e] = sid.emplace(side_key(1), (int32_t)sid.size()).first->second;
    }
    // connected sets of row blocks (ids 0..nr-1) and column blocks (nr..)
    const int32_t nr = (int32_t)rid.size();
    std::vector<int32_t> up(nr + sid.size());
    for (size_t i = 0; i < up.size(); i++) up[i] = (int32_t)i;
    auto root = [&](int32_t x) {
        while (up[x] != x) { up[x] = up[up[x]]; x = up[x]; }
        return x;
    };
    for (size_t e = 0; e < ne; e++) {
        const int32_t a = root(er[e]), b = root(nr + es[e]);
        if (a != b) up[a] = b;
    }
    std::map<int32_t, std::vector<int32_t>> members;
    for (size_t e = 0; e < ne; e++) members[root(er[e])].push_back((int32_t)e);

    int64_t ia[kMaxOrder], ib[kMaxOrder], da[kMaxOrder], db[kMaxOrder], sa[kMaxOrder], sb[kMaxOrder];
    int64_t dc[kMaxOrder];
    for (auto &mb : members) {
        const std::vector<int32_t> &blocks = mb.second;
        if (blocks.size() < 2) continue;
        CrtGroupHost G;
        std::map<int64_t, int32_t> rloc, sloc, kloc;
        std::map<int64_t, int64_t> kext_of;
        bool ok = true;
        double work = 0;
        // keys first (ascending order of each)
        for (int32_t e : blocks) {
            ch.bis.unabs(P.schedule[e], ic);
            rloc.emplace(side_key(0), 0);
            sloc.emplace(side_key(1), 0);
            for (const Pair &p : P.clst[e]) {
                ah.bis.unabs(p.aia, ia);
                ah.bis.block_dims(ia, da);
                int64_t kk = 0, kx = 1;
                for (int d : kdims) { kk = kk * ah.bis.bidims[d] + ia[d]; kx *= da[d]; }
                kloc.emplace(kk, 0);
                kext_of[kk] = kx;
                if (std::fabs(std::fabs(p.tra.coeff) - 1.0) > 0 || std::fabs(std::fabs(p.trb.coeff) - 1.0) > 0) ok = false;
            }
            work += 2.0 * (double)cbt[e].M * (double)cbt[e].N * cbt[e].kflops;
        }
        if (!ok) continue;
        for (auto &x : rloc) { x.second = (int32_t)G.rkey.size(); G.rkey.push_back(x.first); }
        for (auto &x : sloc) { x.second = (int32_t)G.skey.size(); G.skey.push_back(x.first); }
        for (auto &x : kloc) { x.second = (int32_t)G.kkey.size(); G.kkey.push_back(x.first); G.kn.push_back(kext_of[x.first]); }
        G.rn.assign(G.rkey.size(), 0); G.sn.assign(G.skey.size(), 0);
        G.rce.assign(G.rkey.size(), -1); G.sce.assign(G.skey.size(), -1);
        G.cell.assign(G.rkey.size() * G.skey.size(), -1);
        for (int32_t e : blocks) {
            ch.bis.unabs(P.schedule[e], ic);
            ch.bis.block_dims(ic, dc);
            const int32_t R = rloc[side_key(0)], S = sloc[side_key(1)];
            G.rn[R] = cbt[e].M; G.sn[S] = cbt[e].N;
            G.rce[R] = e; G.sce[S] = e;
            G.cell[(size_t)R * G.skey.size() + S] = e;
            for (const Pair &p : P.clst[e]) {
                // the contraction seen from the canonical blocks, as in contract2_tasks
                Perm pa = p.tra.perm, pb = p.trb.perm;
                if (pa.n == 0) pa = Perm::identity(NA);
                if (pb.n == 0) pb = Perm::identity(NB);
                const Perm pinv = pa.inverse();
                Contraction ct = c0;
                ct.permute_a(pinv);
                ct.permute_b(pb.inverse());
                ah.bis.unabs(p.acia, ia); ah.bis.block_dims(ia, da);
                bh.bis.unabs(p.acib, ib); bh.bis.block_dims(ib, db);
                int64_t x = 1;
                for (int i = NA - 1; i >= 0; i--) { sa[i] = x; x *= da[i]; }
                x = 1;
                for (int i = NB - 1; i >= 0; i--) { sb[i] = x; x *= db[i]; }
                int64_t re[kMaxOrder], rs[kMaxOrder], ce[kMaxOrder], cs[kMaxOrder];
                int nra = 0, nrb = 0;
                for (int i = 0; i < NC; i++) {
                    const int64_t t = ct.conn[i];
                    if (t < NC + NA) {
                        if (da[t - NC] != dc[i]) throw error(kErrState, "block extent mismatch (A/C)");
                        re[nra] = dc[i]; rs[nra] = sa[t - NC]; nra++;
                    } else {
                        if (db[t - NC - NA] != dc[i]) throw error(kErrState, "block extent mismatch (B/C)");
                        ce[nrb] = dc[i]; cs[nrb] = sb[t - NC - NA]; nrb++;
                    }
                }
                // contracted dims, ordered by the A dim they stand for
                int64_t ko[kMaxOrder], ke[kMaxOrder], ksa[kMaxOrder], ksb[kMaxOrder];
                int nk = 0;
                for (int i = 0; i < NA; i++) {
                    const int64_t t = ct.conn[NC + i];
                    if (t < NC + NA) continue;
                    if (da[i] != db[t - NC - NA]) throw error(kErrState, "block extent mismatch (A/B)");
                    ko[nk] = pinv.p[i]; ke[nk] = da[i]; ksa[nk] = sa[i]; ksb[nk] = sb[t - NC - NA]; nk++;
                }
                for (int i = 1; i < nk; i++)
                    for (int j = i; j > 0 && ko[j - 1] > ko[j]; j--) {
                        std::swap(ko[j - 1], ko[j]); std::swap(ke[j - 1], ke[j]);
                        std::swap(ksa[j - 1], ksa[j]); std::swap(ksb[j - 1], ksb[j]);
                    }
                ah.bis.unabs(p.aia, ia);
                int64_t kk = 0;
                for (int d : kdims) kk = kk * ah.bis.bidims[d] + ia[d];
                const int32_t K = kloc[kk];
                CrtCell A, B;
                A.off = ah.blk_off[ah.slot_of[p.acia]];
                A.coef = (int32_t)std::lround(p.tra.coeff);
                A.rows = fuse_single(nra, re, rs);
                A.k = fuse_single(nk, ke, ksa);
                B.off = bh.blk_off[bh.slot_of[p.acib]];
                B.coef = (int32_t)std::lround(p.trb.coeff);
                B.rows = fuse_single(nrb, ce, cs);
                B.k = fuse_single(nk, ke, ksb);
                auto ra = G.ac.emplace(std::make_pair(R, K), A);
                auto rb = G.bc.emplace(std::make_pair(K, S), B);
                if ((!ra.second && (ra.first->second.off != A.off || ra.first->second.coef != A.coef)) ||
                    (!rb.second && (rb.first->second.off != B.off || rb.first->second.coef != B.coef)))
                    throw error(kErrState, "one operand cell read from two different blocks");
            }
        }
        // the grouped product must not do much more work than the blocks
        int64_t rows = 0, cols = 0, kt = 0;
        for (int64_t v : G.rn) rows += v;
        for (int64_t v : G.sn) cols += v;
        for (int64_t v : G.kn) kt += round4(v);
        if (2.0 * (double)rows * (double)cols * (double)kt > 1.5 * work) continue;
        if (rows > ((int64_t)1 << 24) || cols > ((int64_t)1 << 24) || kt > ((int64_t)1 << 24)) continue;
        for (int32_t e : blocks) group_of[e] = (int32_t)groups.size();
        groups.push_back(std::move(G));
    }
}

// C placement tables of a group: per row (column) its block and its
// coordinates on the C dims of its side; per C block of the grid its offset
// and C strides (DCrtComp, DCrtCell).
DCrtComp crt_group_tables(const ltg_plan *pl, const BlockTensorHost &ch, const CrtSideMap *sm,
                          const std::vector<CBlockTask> &cbt, const CrtGroupHost &G,
                          std::vector<int32_t> &ctab, std::vector<DCrtCell> &cells) {
    DCrtComp cc;
    cc.rows = 0; cc.cols = 0;
    for (int64_t v : G.rn) cc.rows += (int32_t)v;
    for (int64_t v : G.sn) cc.cols += (int32_t)v;
    cc.ncb = (int32_t)G.skey.size();
    int64_t ic[kMaxOrder], dcb[kMaxOrder], scb[kMaxOrder];
    auto side_entries = [&](int cside, const std::vector<int64_t> &ext, const std::vector<int32_t> &ce) {
        const std::vector<int> &dims = sm[cside].dims;
        for (size_t b = 0; b < ext.size(); b++) {
            ch.bis.unabs(pl->plan().schedule[ce[b]], ic);
            ch.bis.block_dims(ic, dcb);
            for (int64_t i = 0; i < ext[b]; i++) {
                int32_t co[kCrtSideDims] = {0, 0, 0, 0};
                int64_t q = i;
                for (int k = (int)dims.size() - 1; k >= 0; k--) { co[k] = (int32_t)(q % dcb[dims[k]]); q /= dcb[dims[k]]; }
                ctab.push_back((int32_t)b);
                for (int k = 0; k < kCrtSideDims; k++) ctab.push_back(co[k]);
            }
        }
    };
    cc.row_off = (int32_t)ctab.size();
    side_entries(0, G.rn, G.rce);
    cc.col_off = (int32_t)ctab.size();
    side_entries(1, G.sn, G.sce);
    cc.cell_off = (int32_t)ctab.size();
    for (int32_t e : G.cell) {
        if (e < 0) { ctab.push_back(-1); continue; }
        DCrtCell cl;
        std::memset(&cl, 0, sizeof(cl));
        cl.c_off = cbt[e].c_off;
        ch.bis.unabs(pl->plan().schedule[e], ic);
        ch.bis.block_dims(ic, dcb);
        int64_t x = 1;
        for (int d = ch.bis.n - 1; d >= 0; d--) { scb[d] = x; x *= dcb[d]; }
        for (size_t k = 0; k < sm[0].dims.size(); k++) cl.ms[k] = (int32_t)scb[sm[0].dims[k]];
        for (size_t k = 0; k < sm[1].dims.size(); k++) cl.ns[k] = (int32_t)scb[sm[1].dims[k]];
        ctab.push_back((int32_t)cells.size());
        cells.push_back(cl);
    }
    return cc;
}

// Dense layout of one group for the plain path (element offsets in buf, all
// multiples of 4): A panel rows x kt, B panel cols x kt, result rows x cols.
struct PlainGroupLayout {
    int64_t rows = 0, cols = 0, kt = 0, aoff = 0, boff = 0, coff = 0;
    std::vector<int64_t> rofs, sofs, kofs;
};

bool plain_group_layout(const CrtGroupHost &G, int64_t &off, PlainGroupLayout &lay) {
    lay.rofs.clear(); lay.sofs.clear(); lay.kofs.clear();
    lay.rows = lay.cols = lay.kt = 0;
    for (int64_t v : G.rn) { lay.rofs.push_back(lay.rows); lay.rows += v; }
    for (int64_t v : G.sn) { lay.sofs.push_back(lay.cols); lay.cols += v; }
    for (int64_t v : G.kn) { lay.kofs.push_back(lay.kt); lay.kt += round4(v); }
    const int64_t lim = ((int64_t)1 << 31) - 1;
    if (lay.rows * lay.kt > lim || lay.cols * lay.kt > lim || lay.rows * lay.cols > lim) return false;
    auto r4 = [](int64_t x) { return (x + 3) / 4 * 4; };
    lay.aoff = off; off += r4(lay.rows * lay.kt);
    lay.boff = off; off += r4(lay.cols * lay.kt);
    lay.coff = off; off += r4(lay.rows * lay.cols);
    return true;
}

std::vector<std::pair<int64_t, int64_t>> plain_group_shapes(ltg_plan *pl, ltg_bt *c,
                                                           const std::vector<CBlockTask> &cbt,
                                                           std::vector<int32_t> &group_of) {
    std::vector<std::pair<int64_t, int64_t>> shapes;
    group_of.assign(cbt.size(), -1);
    if (!pl->group_products || pl->plan().coalesced) return shapes;
    CrtSideMap sm[2];
    crt_side_maps(pl->plan().contr, c->h, sm);
    std::vector<CrtGroupHost> groups;
    crt_groups(pl, c->h, sm, cbt, groups, group_of);
    int64_t off = 0;
    PlainGroupLayout lay;
    for (const CrtGroupHost &G : groups) {
        if (!plain_group_layout(G, off, lay)) { group_of.assign(cbt.size(), -1); return {}; }
        shapes.push_back({lay.rows, lay.cols});
    }
    return shapes;
}

void external_blocks(const ltg_plan *pl, double ka, double kb, double kc, std::vector<GemmTask> &tasks,
                     std::vector<CBlockTask> &cbt) {
    tasks = pl->ext_tasks;
    for (GemmTask &t : tasks) t.coeff = t.coeff * ka * kb * kc;   // the order contract2_tasks uses
    cbt.clear();
    for (size_t i = 0; i < tasks.size(); i++) {
        if (cbt.empty() || tasks[i].c_off != cbt.back().c_off) {
            CBlockTask b;
            b.c_off = tasks[i].c_off;
            b.t_begin = (int32_t)i;
            b.cm = tasks[i].m; b.cn = tasks[i].n;
            for (int q = 0; q < b.cm.n; q++) b.cm.s0[q] = b.cm.s1[q];
            for (int q = 0; q < b.cn.n; q++) b.cn.s0[q] = b.cn.s1[q];
            b.M = b.cm.total(); b.N = b.cn.total();
            b.coeff0 = tasks[i].coeff;
            cbt.push_back(b);
        }
        CBlockTask &b = cbt.back();
        if (tasks[i].m.total() != b.M || tasks[i].n.total() != b.N)
            throw error(kErrBadArg, "tasks of one C block must share its m and n extents");
        tasks[i].cblk = (int32_t)(cbt.size() - 1);
        b.kflops += (double)tasks[i].k.total();
        b.t_end = (int32_t)i + 1;
    }
}

// ch: the result's space (its block offsets go into the cells); cells_out:
// the cells' host copy, in cell order.
void build_plain_groups(ltg_plan *pl, const BlockTensorHost &ch, const std::vector<CBlockTask> &cbt, double kabc,
                        double post, std::vector<int32_t> &group_of, PlainGroups &pg,
                        std::vector<DCrtCell> *cells_out) {
    CrtSideMap sm[2];
    crt_side_maps(pl->plan().contr, ch, sm);
    std::vector<CrtGroupHost> groups;
    crt_groups(pl, ch, sm, cbt, groups, group_of);
    if (groups.empty()) return;
    std::vector<DGather> pieces;
    std::vector<int4> units;
    std::vector<int2> sunits;
    std::vector<DCrtComp> comps;
    std::vector<int32_t> ctab;
    std::vector<DCrtCell> cells;
    std::vector<int64_t> res_off;
    std::vector<DTask> dt;
    std::vector<DCBlock> dc;
    std::vector<std::vector<std::pair<double, DItem>>> per_cfg(kNumShapes);
    int64_t off = 0;
    PlainGroupLayout lay;
    // one tile shape for all groups (one launch, one tail): that of the
    // costliest group
    int gcfg = -1;
    {
        int64_t o2 = 0;
        double best = -1;
        for (const CrtGroupHost &G : groups) {
            if (!plain_group_layout(G, o2, lay)) { group_of.assign(cbt.size(), -1); return; }
            const double w = (double)lay.rows * lay.cols * lay.kt;
            if (w > best) {
                best = w;
                gcfg = pl->forced_tile >= 0 ? pl->forced_tile : pick_tile(lay.rows, lay.cols);
                auto ov = pl->tile_override.find({lay.rows, lay.cols});
                if (pl->forced_tile < 0 && ov != pl->tile_override.end()) gcfg = ov->second;
            }
        }
    }
    for (size_t gi = 0; gi < groups.size(); gi++) {
        const CrtGroupHost &G = groups[gi];
        if (!plain_group_layout(G, off, lay)) { group_of.assign(cbt.size(), -1); return; }
        auto piece = [&](int src, const CrtCell &cl, int64_t dst_off, int64_t nrow, int64_t K) {
            DGather q;
            std::memset(&q, 0, sizeof(q));
            q.src = src;
            q.src_off = cl.off;
            q.dst_off = dst_off;
            q.rows = (int32_t)nrow;
            q.K = (int32_t)K;
            q.ld = (int32_t)lay.kt;
            q.coef = cl.coef;
            pack_sub(cl.rows, q.nr, q.rext, q.rstr, nullptr);
            pack_sub(cl.k, q.nk, q.kext, q.kstr, nullptr);
            if (cl.rows.total() != nrow || cl.k.total() != K) throw error(kErrState, "grouped cell extents");
            const int32_t ru = (int32_t)std::max<int64_t>(1, std::min<int64_t>(1024, 4096 / std::max<int64_t>(1, K)));
            for (int32_t r0 = 0; r0 < q.rows; r0 += ru)
                units.push_back(make_int4((int32_t)pieces.size(), r0, std::min(ru, q.rows - r0), 0));
            pieces.push_back(q);
        };
        for (const auto &x : G.ac)
            piece(0, x.second, lay.aoff + lay.rofs[x.first.first] * lay.kt + lay.kofs[x.first.second],
                  G.rn[x.first.first], G.kn[x.first.second]);
        for (const auto &x : G.bc)
            piece(1, x.second, lay.boff + lay.sofs[x.first.second] * lay.kt + lay.kofs[x.first.first],
                  G.sn[x.first.second], G.kn[x.first.first]);
        comps.push_back(crt_group_tables(pl, ch, sm, cbt, G, ctab, cells));
        res_off.push_back(lay.coff);
        for (int64_t m = 0; m < lay.rows; m++) sunits.push_back(make_int2((int32_t)gi, (int32_t)m));
        // the dense product: result[m][n] = sum_k A[m][k] B[n][k]
        DTask t;
        std::memset(&t, 0, sizeof(t));
        t.a_off = lay.aoff; t.b_off = lay.boff; t.coeff = 1.0;
        t.K = (int32_t)lay.kt;
        t.nk = 1; t.kext[0] = (int32_t)lay.kt; t.ka_str[0] = 1; t.kb_str[0] = 1;
        t.nm = 1; t.mext[0] = (int32_t)lay.rows; t.ma_str[0] = (int32_t)lay.kt;
        t.nn = 1; t.next[0] = (int32_t)lay.cols; t.nb_str[0] = (int32_t)lay.kt;
        for (int i = 1; i < kDevMaxSub; i++) { t.kext[i] = 1; t.mext[i] = 1; t.next[i] = 1; }
        t.vec_a = 1; t.vec_b = 1;                 // offsets and kt are multiples of 4
        DCBlock b;
        std::memset(&b, 0, sizeof(b));
        b.c_off = lay.coff; b.scale = 1.0;
        b.M = (int32_t)lay.rows; b.N = (int32_t)lay.cols;
        b.nm = 1; b.mext[0] = (int32_t)lay.rows; b.mc_str[0] = (int32_t)lay.cols;
        b.nn = 1; b.next[0] = (int32_t)lay.cols; b.nc_str[0] = 1;
        for (int i = 1; i < kDevMaxSub; i++) { b.mext[i] = 1; b.next[i] = 1; }
        b.t_begin = (int32_t)dt.size(); b.t_end = b.t_begin + 1;
        dt.push_back(t);
        const int cfg = gcfg;
        const int bm = tile_cfg_bm(cfg), bn = tile_cfg_bn(cfg);
        for (int64_t m0 = 0; m0 < lay.rows; m0 += bm)
            for (int64_t n0 = 0; n0 < lay.cols; n0 += bn) {
                DItem it = make_item((int32_t)dc.size(), (int32_t)m0, (int32_t)n0);
                per_cfg[cfg].push_back({(double)bm * bn * (double)lay.kt, it});
            }
        dc.push_back(b);
    }
    std::vector<DItem> items;
    std::vector<DSplit> splits;
    int64_t ws_elems = 0;
    for (int cfg = 0; cfg < kNumShapes; cfg++)
        append_launch(cfg, per_cfg[cfg], dt, dc, pl->ctx->nsm, pl->split_k, items, splits, ws_elems, pg.launches);
    cudaStream_t s = pl->ctx->stream;
    pg.ngroups = (int32_t)groups.size();
    pg.nunits = (int32_t)units.size();
    pg.nsunits = (int32_t)sunits.size();
    pg.scale = kabc * post;
    pg.buf.alloc(std::max<int64_t>(off, 4) * (int64_t)sizeof(double));
    // cells that no pair uses stay zero
    LTG_CUDA(cudaMemsetAsync(pg.buf.p, 0, std::max<int64_t>(off, 4) * sizeof(double), s));
    if (cells_out) *cells_out = cells;
    if (cells.empty()) cells.resize(1);
    upload_vec(pg.pieces, pieces, s);
    upload_vec(pg.units, units, s);
    upload_vec(pg.sunits, sunits, s);
    upload_vec(pg.comps, comps, s);
    upload_vec(pg.res_off, res_off, s);
    upload_vec(pg.ctab, ctab, s);
    upload_vec(pg.cells, cells, s);
    upload_vec(pg.tasks, dt, s);
    upload_vec(pg.cblks, dc, s);
    upload_vec(pg.items, items, s);
    if (!splits.empty()) {
        upload_vec(pg.splits, splits, s);
        pg.ws.alloc(ws_elems * (int64_t)sizeof(double));
    }
}

CrtExec *prepare_crt(ltg_plan *pl, ltg_bt *c, int L, double ka, double kb, double kc, int add, double d) {
    auto key = std::make_tuple(c->uid, ka, kb, kc, add, add ? d : 0.0, L);
    auto it = pl->crt.find(key);
    if (it != pl->crt.end()) return it->second.get();
    if (pl->ctx->capturing) throw error(kErrState, "contraction not prepared before graph capture: call it once outside the capture");
    if (L < 8 || L > kCrtMaxModuli) throw error(kErrBadArg, "modulus count must be 8..16");
    const double kabc = ka * kb * kc;
    if (kabc == 0.0) throw error(kErrUnsupported, "zero contraction coefficient");

    std::vector<GemmTask> tasks;
    std::vector<CBlockTask> cbt;
    contract2_tasks(pl->plan(), pl->a->h, pl->b->h, c->h, ka, kb, kc, tasks, cbt);
    const BlockTensorHost &ch = c->h;
    CrtSideMap sm[2];
    crt_side_maps(pl->plan().contr, ch, sm);
    std::map<int64_t, int64_t> slot_of_off;
    for (size_t sl = 0; sl < ch.blk_off.size(); sl++) slot_of_off[ch.blk_off[sl]] = (int64_t)sl;

    // orientation: the C side with the larger extents goes to the MMA M side
    // (128-row tiles) when that pads less
    double pad_keep = 0, pad_swap = 0;
    for (const CBlockTask &b : cbt) {
        auto padded = [](int64_t x, int64_t y) {
            const int32_t nt = crt_tile_width(y);
            return (double)((x + 127) / 128 * 128) * (double)((y + nt - 1) / nt * nt);
        };
        pad_keep += padded(b.M, b.N);
        pad_swap += padded(b.N, b.M);
    }
    const bool swap = pad_swap < pad_keep;
    // integer coefficients ride on the operand with the smaller arena
    const int coef_src = pl->a->h.total_elems <= pl->b->h.total_elems ? 0 : 1;
    // grouped products of small blocks (their pairs carry coefficients +-1)
    std::vector<CrtGroupHost> groups;
    std::vector<int32_t> group_of(cbt.size(), -1);
    if (pl->group_products && !pl->plan().coalesced) crt_groups(pl, ch, sm, cbt, groups, group_of);

    // panels by (operand, block, row and k mappings, coefficient); one key can
    // hold several panels when the same rows feed different rows of C
    std::map<std::vector<int64_t>, std::vector<int32_t>> pidx;
    std::vector<DCrtPanel> panels;
    std::vector<int32_t> gidx;
    int64_t res_bytes = 0;
    int32_t max_rows = 0;
    std::vector<int32_t> grow;
    // panel of operand src (0: A rows = C side 0, 1: B rows = C side 1)
    auto panel_of = [&](int src, int64_t off, const SubDims &rows, const SubDims &k, bool kb_second, int32_t coef,
                        int64_t c_off) {
        const int side = (src == 1) == swap ? 0 : 1;     // 0: MMA M operand
        std::vector<int64_t> key = {src, off, rows.n, k.n, coef};
        for (int i = 0; i < rows.n; i++) { key.push_back(rows.ext[i]); key.push_back(rows.s0[i]); }
        for (int i = 0; i < k.n; i++) { key.push_back(k.ext[i]); key.push_back(kb_second ? k.s1[i] : k.s0[i]); }
        // global indices of the panel rows, from this C block
        crt_global_index(ch, sm[src], c_off, rows, slot_of_off, grow);
        std::vector<int32_t> &cands = pidx[key];
        for (int32_t id : cands)
            if (std::equal(grow.begin(), grow.end(), gidx.begin() + panels[id].g_off)) return id;
        DCrtPanel p;
        std::memset(&p, 0, sizeof(p));
        p.src = src;
        p.side = side;
        p.src_off = off;
        p.rows = (int32_t)rows.total();
        p.K = (int32_t)k.total();
        p.tr = side == 0 ? 128 : crt_tile_width(p.rows);
        p.rows_pad = (p.rows + p.tr - 1) / p.tr * p.tr;
        p.K_pad = (p.K + 31) / 32 * 32;
        p.coef = coef;
        pack_sub(rows, p.nr, p.rext, p.rstr, nullptr);
        SubDims kk = k;
        if (kb_second) for (int i = 0; i < kk.n; i++) kk.s0[i] = kk.s1[i];
        pack_sub(kk, p.nk, p.kext, p.kstr, nullptr);
        p.res_off = res_bytes;
        res_bytes += ((int64_t)L * p.rows_pad * p.K_pad + 1023) / 1024 * 1024;
        // the padding rows and k of the image stay zero from the buffer's clearing
        p.r0 = 0; p.k0 = 0; p.wrows = p.rows; p.wk = round4(p.K);
        p.g_off = (int32_t)gidx.size();
        gidx.insert(gidx.end(), grow.begin(), grow.end());
        max_rows = std::max(max_rows, p.rows_pad);
        const int32_t id = (int32_t)panels.size();
        panels.push_back(p);
        cands.push_back(id);
        return id;
    };
    std::vector<DCrtTask> dt(tasks.size());
    std::memset(dt.data(), 0, dt.size() * sizeof(DCrtTask));
    int64_t max_sum = 1, max_coef = 1;
    for (size_t e = 0; e < cbt.size(); e++) {
        const CBlockTask &b = cbt[e];
        int64_t sum = 0;
        for (int32_t t = b.t_begin; t < b.t_end; t++) {
            const GemmTask &g = tasks[t];
            const double cr = g.coeff / kabc;
            const int64_t ci = (int64_t)std::llround(cr);
            if (ci == 0 || std::fabs(cr - (double)ci) > 1e-9 || std::llabs(ci) > 64)
                throw error(kErrUnsupported, "modular split precision needs small integer pair coefficients");
            sum += std::llabs(ci) * (int64_t)g.k.total();
            max_coef = std::max<int64_t>(max_coef, std::llabs(ci));
            if (group_of[e] >= 0) continue;          // computed by its grouped product
            const int32_t ca = coef_src == 0 ? (int32_t)ci : 1, cbf = coef_src == 1 ? (int32_t)ci : 1;
            const int32_t pa = panel_of(0, g.a_off, g.m, g.k, false, ca, b.c_off);
            const int32_t pb = panel_of(1, g.b_off, g.n, g.k, true, cbf, b.c_off);
            if (panels[pa].K_pad != panels[pb].K_pad) throw error(kErrState, "panel k extents differ");
            dt[t].px = swap ? pb : pa;
            dt[t].py = swap ? pa : pb;
            dt[t].xres = panels[dt[t].px].res_off;
            dt[t].yres = panels[dt[t].py].res_off;
            dt[t].nkb = panels[pa].K_pad / 32;
            dt[t].pad = 0;
        }
        max_sum = std::max(max_sum, sum);
    }
    // exact INT32 accumulation of |residue| <= 128 products, and the CRT range
    if (max_sum * 128 * 128 >= ((int64_t)1 << 31))
        throw error(kErrUnsupported, "contraction too long for exact modular accumulation");
    double log2M = 0;
    for (int i = 0; i < L; i++) log2M += std::log2((double)kCrtModuli[i]);
    // |c * x * 2^(P - e)| < 2^50 keeps every residue computation exact (the
    // FP64 round-to-integer trick needs magnitudes below 2^51)
    const int pcap = 50 - (int)std::ceil(std::log2((double)max_coef));
    const int P = std::min(pcap, (int)std::floor((log2M - 1.0 - std::log2((double)max_sum)) / 2.0));
    if (P < 24) throw error(kErrUnsupported, "too few moduli for this contraction");

    std::unique_ptr<CrtExec> ex(new CrtExec());
    ex->cp = crt_params(L, P, swap);
    ex->nx = (int32_t)sm[swap ? 1 : 0].size;
    ex->ny = (int32_t)sm[swap ? 0 : 1].size;

    std::vector<DCBlock> dc(cbt.size());
    const double post = (add ? d : 1.0) * kabc;
    for (size_t e = 0; e < cbt.size(); e++) {
        const CBlockTask &b = cbt[e];
        DCBlock &x = dc[e];
        std::memset(&x, 0, sizeof(x));
        x.c_off = b.c_off;
        x.scale = post;
        x.M = (int32_t)b.M; x.N = (int32_t)b.N;
        pack_sub(b.cm, x.nm, x.mext, x.mc_str, nullptr);
        pack_sub(b.cn, x.nn, x.next, x.nc_str, nullptr);
        x.t_begin = b.t_begin; x.t_end = b.t_end;
    }
    // products (one per C block or grouped product), cut into work items below
    struct Prod {
        int32_t cblk, comp, t_begin, t_end, gx, gy, nt;
        int64_t xext, yext;
        double kw;                    // contracted length (work per tile element)
    };
    std::vector<Prod> prods;
    for (size_t e = 0; e < cbt.size(); e++) {
        const CBlockTask &b = cbt[e];
        if (b.t_end <= b.t_begin || group_of[e] >= 0) continue;
        const DCrtTask &t0 = dt[b.t_begin];
        prods.push_back({(int32_t)e, -1, b.t_begin, b.t_end, t0.px, t0.py, panels[t0.py].tr,
                         swap ? b.N : b.M, swap ? b.M : b.N, b.kflops});
    }
    // grouped products: per group one image pair (records, placed after the
    // panels and pieces the split passes process) written cell by cell by
    // pieces, one task and its tiles
    std::vector<DCrtPanel> pieces, records;
    std::vector<DCrtComp> comps;
    std::vector<DCrtCell> cells;
    std::vector<int32_t> ctab;
    size_t npieces = 0;
    for (const CrtGroupHost &G : groups) npieces += G.ac.size() + G.bc.size();
    const int32_t rec_base = (int32_t)(panels.size() + npieces);
    for (size_t gi = 0; gi < groups.size(); gi++) {
        const CrtGroupHost &G = groups[gi];
        std::vector<int32_t> kofs(G.kn.size());
        int32_t kt = 0;
        for (size_t k = 0; k < G.kn.size(); k++) { kofs[k] = kt; kt += round4(G.kn[k]); }
        // one side (0: C rows from A, 1: C columns from B) as an image record
        auto record = [&](int cside, std::vector<int32_t> &ofs) {
            const std::vector<int64_t> &ext = cside == 0 ? G.rn : G.sn;
            const std::vector<int32_t> &ce = cside == 0 ? G.rce : G.sce;
            DCrtPanel r;
            std::memset(&r, 0, sizeof(r));
            r.src = cside;
            r.side = (cside == 1) == swap ? 0 : 1;
            int64_t tot = 0;
            ofs.resize(ext.size());
            for (size_t b = 0; b < ext.size(); b++) { ofs[b] = (int32_t)tot; tot += ext[b]; }
            r.rows = (int32_t)tot;
            r.K = kt;
            r.K_pad = (kt + 31) / 32 * 32;
            r.tr = r.side == 0 ? 128 : crt_tile_width(r.rows);
            r.rows_pad = (r.rows + r.tr - 1) / r.tr * r.tr;
            r.res_off = res_bytes;
            res_bytes += ((int64_t)L * r.rows_pad * r.K_pad + 1023) / 1024 * 1024;
            r.g_off = (int32_t)gidx.size();
            for (size_t b = 0; b < ext.size(); b++) {
                const CBlockTask &cb = cbt[ce[b]];
                crt_global_index(ch, sm[cside], cb.c_off, cside == 0 ? cb.cm : cb.cn, slot_of_off, grow);
                gidx.insert(gidx.end(), grow.begin(), grow.end());
            }
            records.push_back(r);
            return rec_base + (int32_t)records.size() - 1;
        };
        std::vector<int32_t> rofs, sofs;
        const int32_t rrec = record(0, rofs), srec = record(1, sofs);
        const DCrtPanel &RR = records[rrec - rec_base], &SR = records[srec - rec_base];
        auto piece = [&](const DCrtPanel &rec, int src, const CrtCell &cl, int32_t r0, int64_t nrow, int32_t k) {
            DCrtPanel q = rec;
            q.src = src;
            q.src_off = cl.off;
            q.rows = (int32_t)nrow;
            q.K = (int32_t)G.kn[k];
            q.coef = cl.coef;
            q.g_off = rec.g_off + r0;
            pack_sub(cl.rows, q.nr, q.rext, q.rstr, nullptr);
            pack_sub(cl.k, q.nk, q.kext, q.kstr, nullptr);
            if (cl.rows.total() != nrow || cl.k.total() != G.kn[k]) throw error(kErrState, "grouped cell extents");
            q.r0 = r0; q.k0 = kofs[k]; q.wrows = q.rows; q.wk = round4(q.K);
            max_rows = std::max(max_rows, q.wrows);
            pieces.push_back(q);
        };
        for (const auto &x : G.ac) piece(RR, 0, x.second, rofs[x.first.first], G.rn[x.first.first], x.first.second);
        for (const auto &x : G.bc) piece(SR, 1, x.second, sofs[x.first.second], G.sn[x.first.second], x.first.first);
        comps.push_back(crt_group_tables(pl, ch, sm, cbt, G, ctab, cells));
        // the product and its tiles
        const int32_t xrec = swap ? srec : rrec, yrec = swap ? rrec : srec;
        const DCrtPanel &XR = records[xrec - rec_base], &YR = records[yrec - rec_base];
        DCrtTask tk;
        std::memset(&tk, 0, sizeof(tk));
        tk.px = xrec; tk.py = yrec;
        tk.xres = XR.res_off; tk.yres = YR.res_off;
        tk.nkb = XR.K_pad / 32;
        const int32_t ti = (int32_t)dt.size();
        dt.push_back(tk);
        prods.push_back({-1, (int32_t)gi, ti, ti + 1, xrec, yrec, YR.tr, XR.rows, YR.rows, (double)kt});
    }
    // work items: tiles of 256 (two MMA tiles sharing each N-side tile; the
    // default) or 128 rows (one MMA tile; its accumulator slots alternate, so
    // the epilogue of one modulus overlaps the products of the next, but every
    // N-side tile is loaded per 128 rows, which makes the products bound by
    // L2 bandwidth on this part) by nt columns, costliest first
    const int64_t xstep = pl->crt_rows == 128 ? 128 : 256;
    std::vector<std::pair<double, DCrtItem>> iv;
    double total_cost = 0;
    for (const Prod &q : prods)
        for (int64_t x0 = 0; x0 < q.xext; x0 += xstep)
            for (int64_t y0 = 0; y0 < q.yext; y0 += q.nt) {
                DCrtItem it;
                std::memset(&it, 0, sizeof(it));
                it.cblk = q.cblk;
                it.comp = q.comp;
                it.x0 = (int32_t)x0; it.y0 = (int32_t)y0;
                it.nt = q.nt;
                it.nx = xstep == 256 && x0 + 128 < q.xext ? 2 : 1;
                it.t_begin = q.t_begin; it.t_end = q.t_end;
                it.gx = q.gx; it.gy = q.gy;
                iv.push_back({q.kw * q.nt * it.nx, it});
                total_cost += iv.back().first;
            }
    // a 256-row item costing more than one SM's share of the launch is cut
    // into its two 128-row tiles (which load the N-side tile twice), so that
    // no item alone outlasts the others
    const int nsm = std::max(1, pl->ctx->nsm);
    {
        std::vector<std::pair<double, DCrtItem>> cut;
        for (auto &q : iv) {
            if (q.second.nx == 2 && q.first > total_cost / nsm) {
                DCrtItem a = q.second, b = q.second;
                a.nx = b.nx = 1;
                b.x0 += 128;
                cut.push_back({0.5 * q.first, a});
                cut.push_back({0.5 * q.first, b});
            } else {
                cut.push_back(q);
            }
        }
        iv.swap(cut);
    }
    const int32_t nplain = (int32_t)panels.size();                      // panels of their own
    const int32_t nsplit = (int32_t)(panels.size() + pieces.size());   // panels the split passes process
    panels.insert(panels.end(), pieces.begin(), pieces.end());
    panels.insert(panels.end(), records.begin(), records.end());
    if (gidx.size() > ((size_t)1 << 31) - 1 || ctab.size() > ((size_t)1 << 31) - 1)
        throw error(kErrUnsupported, "modular plan index tables too large");

    std::stable_sort(iv.begin(), iv.end(), [](const std::pair<double, DCrtItem> &x, const std::pair<double, DCrtItem> &y) {
        return x.first > y.first;
    });
    std::vector<DCrtItem> items;
    int64_t out_bytes = 0;
    for (auto &q : iv) {
        DCrtItem it = q.second;
        it.res_off = out_bytes;
        out_bytes += (int64_t)L * it.nx * 128 * it.nt;
        items.push_back(it);
    }
    // Each persistent CTA of the products kernel works through its own list:
    // the items, costliest first, dealt in waves of ncta in CTA order (items
    // sharing an operand tile are adjacent in the order, so they run on
    // neighbouring CTAs at the same time and share the tile through L2; with
    // the cut above the waves balance.  Dealing every other wave in reverse
    // order balanced the same on paper and ran the ladder's products 8 %
    // slower).  cta_items holds the ncta + 1 list offsets (into itself), then
    // the lists' item indexes.
    const int32_t ncta = (int32_t)std::min<size_t>(items.size(), (size_t)nsm);
    std::vector<int32_t> cta_items;
    {
        std::vector<std::vector<int32_t>> lists(std::max(ncta, 1));
        for (size_t i = 0; i < items.size(); i++) lists[i % ncta].push_back((int32_t)i);
        cta_items.push_back(ncta + 1);
        for (int32_t b = 0; b < ncta; b++) cta_items.push_back(cta_items.back() + (int32_t)lists[b].size());
        for (int32_t b = 0; b < ncta; b++) cta_items.insert(cta_items.end(), lists[b].begin(), lists[b].end());
    }
    ex->ncta = ncta;
    // every pair of an item shares the tile width of its N operand
    for (const DCrtItem &it : items)
        for (int32_t t = it.t_begin; t < it.t_end; t++)
            if (panels[dt[t].py].tr != it.nt || panels[dt[t].px].tr != 128 || panels[dt[t].px].K_pad != panels[dt[t].py].K_pad)
                throw error(kErrState, "inconsistent tile widths within a C block");

    cudaStream_t s = pl->ctx->stream;
    ex->npanels = nsplit;
    ex->nitems = (int32_t)items.size();
    ex->ngroups = (int32_t)groups.size();
    ex->max_rows = max_rows;
    for (int32_t i = 0; i < nsplit; i++) {
        const DCrtPanel &q = panels[i];
        ex->src_elems += (int64_t)q.rows * q.K;
        ex->res_bytes += (int64_t)L * q.wrows * q.wk;
    }
    // Row families (DCrtFamily): panels of their own (not pieces of grouped
    // images) with one contiguous k run whose global row arrays are equal,
    // such that no other panel feeds those rows.  They are split in one read
    // of the operand (launch_crt_fused); the other panels by the two passes.
    std::vector<char> fused(nsplit, 0);
    std::vector<DCrtFamily> fams;
    std::vector<int32_t> famp, famt;
    std::vector<int4> funits;
    {
        std::vector<int32_t> cnt[2];
        cnt[0].assign(std::max<int32_t>(ex->nx, 1), 0);
        cnt[1].assign(std::max<int32_t>(ex->ny, 1), 0);
        for (int32_t i = 0; i < nsplit; i++) {
            const DCrtPanel &q = panels[i];
            for (int32_t r = 0; r < q.rows; r++) cnt[q.side][gidx[q.g_off + r]]++;
        }
        std::map<std::pair<int32_t, std::vector<int32_t>>, std::vector<int32_t>> byrows;
        for (int32_t i = 0; i < (pl->fused_split ? nplain : 0); i++) {
            const DCrtPanel &q = panels[i];
            if (q.nk != 1 || q.kstr[0] != 1 || q.r0 != 0 || q.k0 != 0 || q.rows <= 0) continue;
            std::vector<int32_t> g(gidx.begin() + q.g_off, gidx.begin() + q.g_off + q.rows);
            byrows[{q.side, g}].push_back(i);
        }
        for (auto &f : byrows) {
            const std::vector<int32_t> &g = f.first.second;
            const int32_t n = (int32_t)f.second.size();
            bool clean = true;
            for (int32_t x : g) if (cnt[f.first.first][x] != n) { clean = false; break; }
            if (!clean) continue;
            DCrtFamily F;
            F.p_begin = (int32_t)famp.size();
            F.rows = (int32_t)g.size();
            int32_t tiles = 0;
            for (int32_t i : f.second) {
                famp.push_back(i);
                famt.push_back(tiles);
                tiles += (panels[i].wk + 15) / 16;
                fused[i] = 1;
                ex->fused_elems += (int64_t)panels[i].rows * panels[i].K;
            }
            F.p_end = (int32_t)famp.size();
            F.ntiles = tiles;
            const int32_t fid = (int32_t)fams.size();
            fams.push_back(F);
            const int32_t fr = crt_fuse_rows(pl->fused_split);
            for (int32_t r0 = 0; r0 < F.rows; r0 += fr)
                funits.push_back(make_int4(fid, r0, std::min<int32_t>(fr, F.rows - r0), 0));
        }
        famt.push_back(0);      // famt[p_end] of the last family is read as a bound only when q + 1 < p_end
    }
    // the other panels' split-pass units: 32 rows of a panel with long k (8
    // threads per row), or about 64 core tiles (8 rows x 16 k, at most 256
    // rows) of one with short k
    std::vector<int4> units;
    for (int32_t i = 0; i < nsplit; i++) {
        if (fused[i]) continue;
        const bool rowmap = panels[i].wk >= 128;
        const int32_t nkt = (panels[i].wk + 15) / 16;
        const int32_t ru = rowmap ? 32 : 8 * std::max(1, std::min(32, 64 / std::max(1, nkt)));
        for (int32_t r0 = 0; r0 < panels[i].wrows; r0 += ru)
            units.push_back(make_int4(i, r0, std::min(ru, panels[i].wrows - r0), rowmap ? 0 : 1));
    }
    ex->nunits = (int32_t)units.size();
    // sampled bounds only where some unit samples (else the exact pass, and
    // no redo launch)
    bool any_sampled = false;
    for (const int4 &u : units) any_sampled = any_sampled || crt_unit_sampled(panels[u.x], u.w);
    ex->sampled = pl->crt_sampled && any_sampled ? 1 : 0;
    for (const int4 &u : units) {
        const DCrtPanel &q = panels[u.x];
        ex->exp_elems += (int64_t)u.z * (ex->sampled && crt_unit_sampled(q, u.w) ? crt_sampled_elems(q) : q.K);
    }
    upload_vec(ex->units, units, s);
    ex->nfunits = (int32_t)funits.size();
    if (!funits.empty()) {
        upload_vec(ex->fams, fams, s);
        upload_vec(ex->famp, famp, s);
        upload_vec(ex->famt, famt, s);
        upload_vec(ex->funits, funits, s);
    }
    ex->res.alloc(std::max<int64_t>(res_bytes, 1024));
    // cells of grouped images that no piece writes stay zero
    LTG_CUDA(cudaMemsetAsync(ex->res.p, 0, std::max<int64_t>(res_bytes, 1024), s));
    ex->out.alloc(std::max<int64_t>(out_bytes, 1024));
    ex->ex.alloc(std::max<int64_t>(ex->nx, 1) * sizeof(int32_t));
    ex->ey.alloc(std::max<int64_t>(ex->ny, 1) * sizeof(int32_t));
    ex->ext.alloc(std::max<int64_t>(ex->nx, 1) * sizeof(int32_t));
    ex->eyt.alloc(std::max<int64_t>(ex->ny, 1) * sizeof(int32_t));
    upload_vec(ex->panels, panels, s);
    upload_vec(ex->tasks, dt, s);
    upload_vec(ex->items, items, s);
    upload_vec(ex->cta_items, cta_items, s);
    upload_vec(ex->cblks, dc, s);
    upload_vec(ex->gidx, gidx, s);
    ex->cells_host = cells;
    if (comps.empty()) comps.resize(1);
    if (ctab.empty()) ctab.resize(1);
    if (cells.empty()) cells.resize(1);
    upload_vec(ex->comps, comps, s);
    upload_vec(ex->ctab, ctab, s);
    upload_vec(ex->cells, cells, s);
    ex->scale = post;
    std::vector<char> in_sched(c->h.blk_abs.size(), 0);
    for (int64_t cabs : pl->plan().schedule) {
        int64_t sl = c->h.slot_of[cabs];
        in_sched[sl] = 1;
        ex->sched_slots.push_back(sl);
    }
    for (size_t sl = 0; sl < in_sched.size(); sl++) {
        if (in_sched[sl]) continue;
        int64_t b0 = c->h.blk_off[sl], b1 = b0 + c->h.blk_size[sl];
        if (!ex->zero_ranges.empty() && ex->zero_ranges.back().second >= b0 - 3) ex->zero_ranges.back().second = b1;
        else ex->zero_ranges.push_back({b0, b1});
    }
    LTG_CUDA(cudaStreamSynchronize(s));
    CrtExec *raw = ex.get();
    pl->crt[key] = std::move(ex);
    return raw;
}

// ------------------------------------------------------------ transfers

// Every address a transfer/dot job can form must lie inside its arena.
void validate_transfer(const TransferPlan &plan, const std::vector<int64_t> &src_sizes, int64_t dst_size) {
    for (const TJob &j : plan.jobs) {
        int64_t n = 1;
        for (int d = 0; d < j.ndim; d++) n *= j.ext[d];
        if (dst_size >= 0 && (j.dst_off < 0 || j.dst_off + n > dst_size))
            throw error(kErrState, "transfer destination outside its arena");
        for (int t = 0; t < j.nterms; t++) {
            const TTerm &tm = plan.terms[j.term0 + t];
            int64_t m = tm.src_off;
            for (int d = 0; d < j.ndim; d++) m += (int64_t)(j.ext[d] - 1) * tm.sstr[d];
            if (tm.src < 0 || tm.src >= (int)src_sizes.size() || tm.src_off < 0 || m >= src_sizes[tm.src])
                throw error(kErrState, "transfer source outside its arena");
        }
    }
    for (const TUnit &u : plan.units)
        if (u.job < 0 || u.job >= (int32_t)plan.jobs.size()) throw error(kErrState, "bad transfer unit");
}

// Cached copy/add plans: the first call for a given (operands, permutations,
// coefficients, destination, mode) builds and uploads the task arrays; later
// calls, including calls inside a CUDA-graph capture, only launch.
// Device form of a transfer plan: every job seen as planes of A rows x B
// columns (DJob).  Jobs whose terms all read the columns with unit stride run
// in row mode (warp items of about kItemElems elements: row chunks x column
// segments); a job
// with a transposing term runs in tiled mode, tiles of at most 64x64 whose
// transposing terms are staged through shared memory.  Units hold about
// kTransferUnitElems elements.
struct DeviceTransfer {
    std::vector<DJob> jobs;
    std::vector<DTerm> terms;
    std::vector<DUnit> units;          // row-mode units, then tiled-mode units
    int32_t nrow = 0, ntiled = 0;
    int32_t max_terms = 0, tile_bytes = 0;
};
constexpr int64_t kTransferUnitElems = 32768;
constexpr int32_t kItemElems = 4096;       // row mode: elements per warp item (about)
constexpr int32_t kTileSide = 64;          // largest tile side (elements)
constexpr int64_t kTileSmemDoubles = 12288; // tiled mode: shared memory for all terms' tiles (96 KiB)

DeviceTransfer device_transfer(const TransferPlan &plan, int64_t unit_elems = kTransferUnitElems) {
    DeviceTransfer o;
    std::vector<DUnit> tiled_units;
    for (const TJob &j : plan.jobs) {
        const int n = j.ndim, L = n - 1;
        const TTerm *T = plan.terms.data() + j.term0;
        // Row dim q: the destination dim that is contiguous in the first
        // source whose innermost stride is not 1 (a transposition), else the
        // next-to-innermost dim.
        int q = -1;
        bool transposing = false;
        if (n >= 2) {
            q = L - 1;
            for (int t = 0; t < j.nterms; t++) {
                if (T[t].sstr[L] == 1) continue;
                transposing = true;
                for (int d = 0; d < L; d++)
                    if (T[t].sstr[d] == 1) { q = d; break; }
                break;
            }
        }
        int64_t dstr[kMaxOrder];
        int64_t acc = 1;
        for (int d = n - 1; d >= 0; d--) { dstr[d] = acc; acc *= j.ext[d]; }
        DJob dj{};
        dj.dst_off = j.dst_off;
        dj.nterms = j.nterms;
        dj.term0 = (int32_t)o.terms.size();
        dj.A = q >= 0 ? j.ext[q] : 1;
        dj.B = j.ext[L];
        dj.dq = q >= 0 ? (int32_t)dstr[q] : 0;
        for (int d = 0; d < L; d++) {
            if (d == q) continue;
            dj.oext[dj.nout] = j.ext[d];
            dj.odst[dj.nout] = (int32_t)dstr[d];
            dj.nout++;
        }
        dj.tiled = transposing ? 1 : 0;
        dj.seg = dj.B > kItemElems ? kItemElems : dj.B;
        dj.nseg = (dj.B + dj.seg - 1) / dj.seg;
        dj.ra = std::max<int32_t>(1, std::min<int32_t>(dj.A, kItemElems / dj.seg));
        dj.nra = (dj.A + dj.ra - 1) / dj.ra;
        bool vec = !transposing && dj.seg % 2 == 0 && dj.B % 2 == 0 && dj.dst_off % 2 == 0 && dj.dq % 2 == 0;
        for (int k = 0; k < dj.nout; k++) vec = vec && dj.odst[k] % 2 == 0;
        // tiled mode: square-ish tiles of at most kTileSide whose tiles of all
        // terms fit kTileSmemDoubles; balanced tile extents per dim
        int32_t side = kTileSide;
        while (side > 8 && (int64_t)std::max(1, j.nterms) * side * (side + 1) > kTileSmemDoubles) side--;
        dj.nta = (dj.A + side - 1) / side;
        dj.ntb = (dj.B + side - 1) / side;
        const int32_t ta_ext = (dj.A + dj.nta - 1) / dj.nta, tb_ext = (dj.B + dj.ntb - 1) / dj.ntb;
        int32_t toff = 0;
        for (int t = 0; t < j.nterms; t++) {
            DTerm dt{};
            dt.src_off = T[t].src_off;
            dt.coeff = T[t].coeff;
            dt.src = T[t].src;
            dt.sq = q >= 0 ? T[t].sstr[q] : 0;
            dt.sb = T[t].sstr[L];
            if (transposing) {
                dt.tmode = dt.sb == 1 ? 0 : 1;
                dt.tld = dt.tmode == 0 ? tb_ext : ta_ext + 1;
                toff += toff & 1;                        // 16-byte aligned tiles
                dt.toff = toff;
                toff += dt.tmode == 0 ? ta_ext * tb_ext : tb_ext * (ta_ext + 1);
                // 16-byte copies along the columns: every tile row starts even
                dt.tvec = dt.tmode == 0 && tb_ext % 2 == 0 && dj.B % 2 == 0 && dt.src_off % 2 == 0 &&
                          dt.sq % 2 == 0 ? 1 : 0;
            }
            int k = 0;
            for (int d = 0; d < L; d++)
                if (d != q) dt.osrc[k++] = T[t].sstr[d];
            vec = vec && dt.sb == 1 && dt.src_off % 2 == 0 && dt.sq % 2 == 0;
            for (int kk = 0; kk < dj.nout; kk++) {
                vec = vec && dt.osrc[kk] % 2 == 0;
                if (dt.osrc[kk] % 2) dt.tvec = 0;
            }
            o.terms.push_back(dt);
        }
        dj.vec = vec ? 1 : 0;
        o.max_terms = std::max(o.max_terms, j.nterms);
        if (transposing) o.tile_bytes = std::max<int32_t>(o.tile_bytes, (toff + 1) * (int32_t)sizeof(double));
        const int32_t ji = (int32_t)o.jobs.size();
        o.jobs.push_back(dj);
        int64_t planes = 1;
        for (int k = 0; k < dj.nout; k++) planes *= dj.oext[k];
        if (planes * dj.A * (int64_t)dj.B >= (int64_t(1) << 31))
            throw error(kErrUnsupported, "block too large for one transfer job");
        int64_t items, per_unit;
        if (dj.tiled) {
            items = planes * dj.nta * dj.ntb;
            const int64_t tile = (int64_t)((dj.A + dj.nta - 1) / dj.nta) * ((dj.B + dj.ntb - 1) / dj.ntb);
            per_unit = std::max<int64_t>(1, unit_elems / tile);
        } else {
            items = planes * dj.nra * dj.nseg;
            const int64_t item = (int64_t)dj.ra * dj.seg;
            per_unit = std::max<int64_t>(8, (unit_elems / item + 7) / 8 * 8);
        }
        for (int64_t r = 0; r < items; r += per_unit) {
            DUnit u{};
            u.job = ji;
            u.row_begin = r;
            u.row_end = std::min(items, r + per_unit);
            (dj.tiled ? tiled_units : o.units).push_back(u);
        }
    }
    o.nrow = (int32_t)o.units.size();
    o.ntiled = (int32_t)tiled_units.size();
    o.units.insert(o.units.end(), tiled_units.begin(), tiled_units.end());
    return o;
}

struct TransferExec {
    DevBuf jobs, terms, units, srcs;
    int32_t nrow = 0, ntiled = 0, max_terms = 0, tile_bytes = 0;
    std::vector<char> dst_nonzero;
};
typedef std::tuple<std::vector<const ltg_bt *>, std::vector<int8_t>, std::vector<double>,
                   const ltg_bt *, int, double> transfer_key;
std::mutex g_tr_mtx;
std::map<transfer_key, std::unique_ptr<TransferExec>> g_tr_cache;


void run_transfer(ltg_ctx *ctx, const std::vector<ltg_bt *> &srcs, const std::vector<Perm> &perms,
                  const std::vector<double> &coeffs, ltg_bt *dst, bool add, double d) {
    transfer_key key;
    for (size_t t = 0; t < srcs.size(); t++) {
        if (srcs[t]->ctx != ctx) throw error(kErrBadArg, "operands belong to different contexts");
        std::get<0>(key).push_back(srcs[t]);
        for (int i = 0; i < perms[t].n; i++) std::get<1>(key).push_back(perms[t].p[i]);
    }
    std::get<2>(key) = coeffs;
    std::get<3>(key) = dst;
    std::get<4>(key) = add ? 1 : 0;
    std::get<5>(key) = add ? d : 0.0;
    TransferExec *ex = nullptr;
    cudaStream_t s = ctx->stream;
    {
        std::lock_guard<std::mutex> lk(g_tr_mtx);
        auto it = g_tr_cache.find(key);
        if (it != g_tr_cache.end()) ex = it->second.get();
    }
    if (!ex) {
        if (ctx->capturing) throw error(kErrState, "copy/add not prepared before graph capture: call it once outside the capture");
        std::vector<TransferTerm> terms;
        for (size_t t = 0; t < srcs.size(); t++)
            terms.push_back(TransferTerm{&srcs[t]->h, perms[t], coeffs[t], (int32_t)t});
        TransferPlan plan;
        plan_transfer(terms, dst->h, add, plan);
        std::vector<int64_t> ssz;
        for (ltg_bt *b : srcs) ssz.push_back(b->h.total_elems);
        validate_transfer(plan, ssz, dst->h.total_elems);
        std::unique_ptr<TransferExec> nx(new TransferExec());
        DeviceTransfer dt = device_transfer(plan);
        upload_vec(nx->jobs, dt.jobs, s);
        upload_vec(nx->terms, dt.terms, s);
        upload_vec(nx->units, dt.units, s);
        std::vector<const double *> sp;
        for (ltg_bt *b : srcs) sp.push_back(b->arena.as<double>());
        upload_vec(nx->srcs, sp, s);
        nx->nrow = dt.nrow;
        nx->ntiled = dt.ntiled;
        nx->max_terms = dt.max_terms;
        nx->tile_bytes = dt.tile_bytes;
        nx->dst_nonzero = plan.dst_nonzero;
        ex = nx.get();
        std::lock_guard<std::mutex> lk(g_tr_mtx);
        g_tr_cache[key] = std::move(nx);
    }
    TimedLaunch tl(ctx, LTG_KERNEL_TRANSFER);
    LTG_CUDA(launch_transfer(ex->jobs.as<DJob>(), ex->terms.as<DTerm>(), ex->units.as<DUnit>(),
                             ex->nrow, ex->ntiled, ex->max_terms, ex->tile_bytes, ex->srcs.as<const double *>(), dst->arena.as<double>(),
                             add ? 1 : 0, d, s));
    tl.done();
    ctx->launches++;
    for (size_t sl = 0; sl < ex->dst_nonzero.size(); sl++)
        dst->h.nonzero[sl] = add ? (dst->h.nonzero[sl] || ex->dst_nonzero[sl]) : ex->dst_nonzero[sl];
}

void forget_transfer(const ltg_bt *t) {
    std::lock_guard<std::mutex> lk(g_tr_mtx);
    for (auto it = g_tr_cache.begin(); it != g_tr_cache.end();) {
        const auto &v = std::get<0>(it->first);
        bool hit = std::get<3>(it->first) == t || std::find(v.begin(), v.end(), t) != v.end();
        if (hit) it = g_tr_cache.erase(it);
        else ++it;
    }
}

// Cached dot-product plans so that repeated (and graph-captured) calls issue
// only kernel launches.
struct DotExec {
    DevBuf jobs, terms, units, partials;
    int32_t nrow = 0, ntiled = 0, tile_bytes = 0;
};
std::mutex g_dot_mtx;
std::map<std::tuple<const ltg_bt *, const ltg_bt *, std::vector<int8_t>, std::vector<int8_t>>,
         std::unique_ptr<DotExec>> g_dot_cache;

DotExec *prepare_dot(ltg_bt *a, const Perm &pa, ltg_bt *b, const Perm &pb) {
    std::vector<int8_t> ka(pa.p, pa.p + pa.n), kb(pb.p, pb.p + pb.n);
    auto key = std::make_tuple((const ltg_bt *)a, (const ltg_bt *)b, ka, kb);
    std::lock_guard<std::mutex> lk(g_dot_mtx);
    auto it = g_dot_cache.find(key);
    if (it != g_dot_cache.end()) return it->second.get();
    if (a->ctx->capturing) throw error(kErrState, "dot product not prepared before graph capture");
    TransferPlan plan;
    plan_dot(a->h, pa, b->h, pb, plan);
    validate_transfer(plan, {a->h.total_elems, b->h.total_elems}, -1);
    std::unique_ptr<DotExec> ex(new DotExec());
    cudaStream_t s = a->ctx->stream;
    // larger units for the dot product: each unit ends in a CTA reduction
    DeviceTransfer dt = device_transfer(plan, 4 * kTransferUnitElems);
    upload_vec(ex->jobs, dt.jobs, s);
    upload_vec(ex->terms, dt.terms, s);
    upload_vec(ex->units, dt.units, s);
    ex->partials.alloc(std::max<size_t>(dt.units.size(), 1) * sizeof(double));
    ex->nrow = dt.nrow;
    ex->ntiled = dt.ntiled;
    ex->tile_bytes = dt.tile_bytes;
    DotExec *raw = ex.get();
    g_dot_cache[key] = std::move(ex);
    return raw;
}

void forget_dot(const ltg_bt *t) {
    std::lock_guard<std::mutex> lk(g_dot_mtx);
    for (auto it = g_dot_cache.begin(); it != g_dot_cache.end();) {
        if (std::get<0>(it->first) == t || std::get<1>(it->first) == t) it = g_dot_cache.erase(it);
        else ++it;
    }
}

// LTG_TASK_WORDS int64 per task (layout in ltg.h)
void pack_task(const GemmTask &t, int64_t *w) {
    std::memset(w, 0, LTG_TASK_WORDS * sizeof(int64_t));
    w[0] = t.c_off; w[1] = t.a_off; w[2] = t.b_off;
    const SubDims *sd[3] = {&t.m, &t.n, &t.k};
    for (int g = 0; g < 3; g++) {
        int64_t *x = w + 3 + 13 * g;
        x[0] = sd[g]->n;
        for (int i = 0; i < sd[g]->n; i++) { x[1 + 3 * i] = sd[g]->ext[i]; x[2 + 3 * i] = sd[g]->s0[i]; x[3 + 3 * i] = sd[g]->s1[i]; }
    }
    std::memcpy(&w[42], &t.coeff, sizeof(double));
}
GemmTask unpack_task(const int64_t *w) {
    GemmTask t;
    t.c_off = w[0]; t.a_off = w[1]; t.b_off = w[2];
    SubDims *sd[3] = {&t.m, &t.n, &t.k};
    for (int g = 0; g < 3; g++) {
        const int64_t *x = w + 3 + 13 * g;
        if (x[0] < 0 || x[0] > kMaxSub) throw error(kErrBadArg, "task: sub-dimension count out of range");
        sd[g]->n = (int)x[0];
        for (int i = 0; i < sd[g]->n; i++) {
            if (x[1 + 3 * i] < 1 || x[1 + 3 * i] > ((int64_t)1 << 30)) throw error(kErrBadArg, "task: extent out of range");
            // the kernels hold strides as int32
            if (x[2 + 3 * i] < 0 || x[3 + 3 * i] < 0 || x[2 + 3 * i] > INT32_MAX || x[3 + 3 * i] > INT32_MAX)
                throw error(kErrBadArg, "task: stride out of range");
            sd[g]->ext[i] = (int32_t)x[1 + 3 * i]; sd[g]->s0[i] = x[2 + 3 * i]; sd[g]->s1[i] = x[3 + 3 * i];
            if (sd[g]->total() > ((int64_t)1 << 31) - 1) throw error(kErrBadArg, "task: dimension too large");
        }
    }
    std::memcpy(&t.coeff, &w[42], sizeof(double));
    t.cblk = 0;
    return t;
}

}  // namespace

extern "C" {

const char *ltg_last_error(void) { return g_last_error.c_str(); }
int ltg_version(void) { return 100; }

// Device-wait errors.  A tcgen05 kernel whose pipeline wait gave up sets the
// context's error word (7) and unwinds; the word is copied to pinned host
// memory after each such launch (outside graph capture) and reported as
// LTG_ERR_TIMEOUT by the next contraction call or by ltg_ctx_synchronize,
// which then clear it.
static void fetch_device_wait(ltg_ctx *ctx) {
    if (!ctx->capturing)
        LTG_CUDA(cudaMemcpyAsync(ctx->wait_err_host, ctx->wait_err.p, sizeof(int32_t), cudaMemcpyDeviceToHost,
                                 ctx->stream));
}

static void report_device_wait(ltg_ctx *ctx) {
    if (*ctx->wait_err_host == 0) return;
    // every copy of the word still in flight lands before it is cleared
    LTG_CUDA(cudaStreamSynchronize(ctx->stream));
    LTG_CUDA(cudaMemsetAsync(ctx->wait_err.p, 0, sizeof(int32_t), ctx->stream));
    LTG_CUDA(cudaStreamSynchronize(ctx->stream));
    *ctx->wait_err_host = 0;
    throw error(kErrTimeout, "a bounded device wait of a split-precision products kernel gave up (limit " +
                                 std::to_string(ctx->wait_ns) + " ns); its results are invalid");
}

int ltg_ctx_create(int device, ltg_ctx **out) {
    return guard([&] {
        if (!out) throw error(kErrBadArg, "null output");
        std::unique_ptr<ltg_ctx> c(new ltg_ctx());
        c->device = device;
        // device < 0: host-only context (schedules, orbits and host fills;
        // no device memory, every device operation returns LTG_ERR_STATE).
        if (device >= 0) {
            LTG_CUDA(cudaSetDevice(device));
            LTG_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
            LTG_CUDA(cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device));
            c->scratch_counter.alloc(64 * sizeof(int32_t));
            c->dot_out.alloc(sizeof(double));
            c->wait_err.alloc(sizeof(int32_t));
            LTG_CUDA(cudaMemset(c->wait_err.p, 0, sizeof(int32_t)));
            LTG_CUDA(cudaMallocHost(&c->wait_err_host, sizeof(int32_t)));
            *c->wait_err_host = 0;
        }
        unsigned hc = std::thread::hardware_concurrency();
        c->host_threads = hc ? (int)hc : 1;
        *out = c.release();
    });
}

int ltg_ctx_destroy(ltg_ctx *ctx) {
    return guard([&] {
        check_ctx(ctx);
        if (ctx->device >= 0) {
            cudaStreamSynchronize(ctx->stream);
            for (auto &p : ctx->timing.pending) {
                cudaEventDestroy(std::get<1>(p));
                cudaEventDestroy(std::get<2>(p));
            }
            for (cudaEvent_t e : ctx->timing.pool) cudaEventDestroy(e);
            cudaStreamDestroy(ctx->stream);
            if (ctx->wait_err_host) cudaFreeHost(ctx->wait_err_host);
        }
        delete ctx;
    });
}

int ltg_ctx_synchronize(ltg_ctx *ctx) {
    return guard([&] {
        check_ctx(ctx);
        if (ctx->device < 0) return;
        fetch_device_wait(ctx);
        LTG_CUDA(cudaStreamSynchronize(ctx->stream));
        if (!ctx->capturing) report_device_wait(ctx);
    });
}

int ltg_ctx_set_wait_limit(ltg_ctx *ctx, uint64_t ns) {
    return guard([&] { check_ctx(ctx); ctx->wait_ns = ns; });
}

int ltg_ctx_wait_limit(ltg_ctx *ctx, uint64_t *ns) {
    return guard([&] { check_ctx(ctx); if (!ns) throw error(kErrBadArg, "null output"); *ns = ctx->wait_ns; });
}

int ltg_ctx_stream(ltg_ctx *ctx, void **stream) {
    return guard([&] { check_ctx(ctx); if (!stream) throw error(kErrBadArg, "null output"); *stream = ctx->stream; });
}

int ltg_ctx_set_host_threads(ltg_ctx *ctx, int nthreads) {
    return guard([&] { check_ctx(ctx); ctx->host_threads = nthreads < 1 ? 1 : nthreads; });
}

int ltg_ctx_launch_count(ltg_ctx *ctx, int64_t *count) {
    return guard([&] { check_ctx(ctx); if (!count) throw error(kErrBadArg, "null output"); *count = ctx->launches; });
}

int ltg_ctx_set_timing(ltg_ctx *ctx, int32_t enable) {
    return guard([&] {
        check_ctx(ctx);
        need_dev(ctx);
        collect_timing(ctx);
        ctx->timing.enabled = enable != 0;
        if (enable)
            for (int k = 0; k < LTG_KERNEL_KINDS; k++) { ctx->timing.ms[k] = 0.0; ctx->timing.count[k] = 0; }
    });
}

int ltg_ctx_kernel_times(ltg_ctx *ctx, double *ms, int64_t *launches) {
    return guard([&] {
        check_ctx(ctx);
        need_dev(ctx);
        if (!ms || !launches) throw error(kErrBadArg, "null output");
        collect_timing(ctx);
        for (int k = 0; k < LTG_KERNEL_KINDS; k++) { ms[k] = ctx->timing.ms[k]; launches[k] = ctx->timing.count[k]; }
    });
}

int ltg_bt_create(ltg_ctx *ctx, const ltg_bt_spec *spec, ltg_bt **out) {
    return guard([&] {
        check_ctx(ctx);
        if (!out) throw error(kErrBadArg, "null output");
        std::unique_ptr<ltg_bt> bt(new ltg_bt());
        bt->ctx = ctx;
        parse_spec(spec, bt->h);
        alloc_arena(bt.get());
        *out = bt.release();
    });
}

int ltg_bt_create_permuted(ltg_bt *a, const int32_t *perm, ltg_bt **out) {
    return guard([&] {
        check_bt(a);
        if (!out) throw error(kErrBadArg, "null output");
        std::unique_ptr<ltg_bt> bt(new ltg_bt());
        bt->ctx = a->ctx;
        Perm p = perm_from(a->h.bis.n, perm);
        permute_space(a->h.bis, a->h.sym, p, bt->h.bis, bt->h.sym);
        alloc_arena(bt.get());
        *out = bt.release();
    });
}

namespace {
bool same_part(const SePart &x, const SePart &y, int n) {
    for (int d = 0; d < n; d++)
        if (x.pdims[d] != y.pdims[d] || x.bipdims[d] != y.bipdims[d]) return false;
    return x.forbidden == y.forbidden;
}
bool same_label(const SeLabel &x, const SeLabel &y, int n) {
    if (x.nirrep != y.nirrep || x.rule.size() != y.rule.size()) return false;
    for (int d = 0; d < n; d++) if (x.labels[d] != y.labels[d]) return false;
    for (size_t i = 0; i < x.rule.size(); i++) {
        if (x.rule[i].size() != y.rule[i].size()) return false;
        for (size_t k = 0; k < x.rule[i].size(); k++) {
            if (x.rule[i][k].intr != y.rule[i][k].intr) return false;
            for (int d = 0; d < n; d++) if (x.rule[i][k].seq[d] != y.rule[i][k].seq[d]) return false;
        }
    }
    return true;
}
}  // namespace

int ltg_bt_create_sum_space(int32_t nterms, ltg_bt *const *a, const int32_t *perms, ltg_bt **out) {
    return guard([&] {
        if (nterms < 1 || !a || !out) throw error(kErrBadArg, "a sum needs at least one term");
        for (int32_t t = 0; t < nterms; t++) check_bt(a[t]);
        const int n = a[0]->h.bis.n;
        std::vector<Bis> bis(nterms);
        std::vector<Symmetry> sym(nterms);
        for (int32_t t = 0; t < nterms; t++) {
            if (a[t]->h.bis.n != n) throw error(kErrBadDims, "terms of different order");
            permute_space(a[t]->h.bis, a[t]->h.sym, perm_from(n, perms ? perms + (size_t)t * n : nullptr),
                          bis[t], sym[t]);
            if (!bis[t].equals(bis[0])) throw error(kErrBadDims, "terms of a sum with different block index spaces");
        }
        std::unique_ptr<ltg_bt> bt(new ltg_bt());
        bt->ctx = a[0]->ctx;
        bt->h.bis = bis[0];
        // permutational elements in every term's group (with the same sign)
        std::vector<SePerm> common = perm_group_closure(n, sym[0].perm);
        for (int32_t t = 1; t < nterms; t++) {
            const std::vector<SePerm> g = perm_group_closure(n, sym[t].perm);
            std::vector<SePerm> keep;
            for (const SePerm &e : common)
                for (const SePerm &f : g)
                    if (e.perm == f.perm && e.coeff == f.coeff) { keep.push_back(e); break; }
            common.swap(keep);
        }
        for (const SePerm &e : common)
            if (!e.perm.is_identity()) bt->h.sym.perm.push_back(e);
        // partition and label rules shared by all terms
        bool parts = true, labels = true;
        for (int32_t t = 1; t < nterms; t++) {
            parts = parts && sym[t].part.size() == sym[0].part.size();
            for (size_t i = 0; parts && i < sym[0].part.size(); i++) parts = same_part(sym[0].part[i], sym[t].part[i], n);
            labels = labels && sym[t].label.size() == sym[0].label.size();
            for (size_t i = 0; labels && i < sym[0].label.size(); i++)
                labels = same_label(sym[0].label[i], sym[t].label[i], n);
        }
        if (parts) bt->h.sym.part = sym[0].part;
        if (labels) bt->h.sym.label = sym[0].label;
        alloc_arena(bt.get());
        *out = bt.release();
    });
}

namespace {
// The symmetrizer's group: nidx 2, indexes idx[0] and idx[1]: {e, (i1 i2)};
// nidx -1, a unitary permutation idx[0..n): {e, P}; nidx 4: the 24
// permutations of indexes idx[0..3].  Signs: +1 (symm), else the parity.
std::vector<SePerm> symmetrizer_group(int n, int32_t nidx, const int32_t *idx, bool symm) {
    if (!idx) throw error(kErrBadArg, "null symmetrizer indexes");
    std::vector<SePerm> g;
    SePerm e;
    e.perm = Perm::identity(n);
    e.coeff = 1.0;
    if (nidx == 2 || nidx == -1) {
        SePerm q = e;
        if (nidx == 2) {
            if (idx[0] < 0 || idx[0] >= n || idx[1] < 0 || idx[1] >= n || idx[0] == idx[1])
                throw error(kErrBadArg, "symmetrizer indexes out of range");
            std::swap(q.perm.p[idx[0]], q.perm.p[idx[1]]);
        } else {
            q.perm = perm_from(n, idx);
            Perm sq = q.perm;
            sq.permute(q.perm);
            if (!sq.is_identity() || q.perm.is_identity())
                throw error(kErrBadArg, "the symmetrizer permutation must be its own inverse");
        }
        q.coeff = symm ? 1.0 : -1.0;
        g.push_back(e);
        g.push_back(q);
        return g;
    }
    if (nidx != 4) throw error(kErrBadArg, "a symmetrizer takes 2 or 4 indexes or a permutation");
    for (int k = 0; k < 4; k++) {
        if (idx[k] < 0 || idx[k] >= n) throw error(kErrBadArg, "symmetrizer indexes out of range");
        for (int l = 0; l < k; l++) if (idx[k] == idx[l]) throw error(kErrBadArg, "repeated symmetrizer index");
    }
    int pi[4] = {0, 1, 2, 3};
    do {
        SePerm q = e;
        for (int k = 0; k < 4; k++) q.perm.p[idx[k]] = (int8_t)idx[pi[k]];
        int inv = 0;
        for (int a = 0; a < 4; a++) for (int b = a + 1; b < 4; b++) if (pi[a] > pi[b]) inv++;
        q.coeff = symm || inv % 2 == 0 ? 1.0 : -1.0;
        g.push_back(q);
    } while (std::next_permutation(pi, pi + 4));
    return g;
}

// Every block's allowedness is unchanged by the permutation.
bool allowed_invariant(const Bis &bis, const Symmetry &sym, const Perm &p) {
    int64_t bidx[kMaxOrder], pb[kMaxOrder];
    const int64_t nb = bis.nblocks();
    for (int64_t a = 0; a < nb; a++) {
        bis.unabs(a, bidx);
        for (int d = 0; d < bis.n; d++) pb[d] = bidx[p.p[d]];
        if (sym.is_allowed(bis.n, bidx) != sym.is_allowed(bis.n, pb)) return false;
    }
    return true;
}
}  // namespace

namespace {

// The space of S-sums of a tensor with block index space bis and symmetry
// sym: bis with S's generators, the elements of sym's group that map S onto
// itself, and sym's partition and label rules if S leaves them unchanged.
void symmetrized_space(const Bis &bis, const Symmetry &sym, int32_t nidx, const int32_t *idx, int32_t symm,
                       BlockTensorHost &h) {
    const int n = bis.n;
    const std::vector<SePerm> S = symmetrizer_group(n, nidx, idx, symm != 0);
    for (const SePerm &g : S)
        if (!bis.permuted(g.perm).equals(bis))
            throw error(kErrBadDims, "symmetrized indexes with different block structure");
    h.bis = bis;
    // generators of the symmetrizer's group
    if (nidx == 4) {
        for (int k = 1; k < 4; k++) {
            SePerm q;
            q.perm = Perm::identity(n);
            std::swap(q.perm.p[idx[0]], q.perm.p[idx[k]]);
            q.coeff = symm ? 1.0 : -1.0;
            h.sym.perm.push_back(q);
        }
    } else {
        h.sym.perm.push_back(S[1]);
    }
    // the operand's elements that map the symmetrizer's group onto itself
    // (h S h^-1 = S) remain symmetries of the sum over S
    for (const SePerm &x : perm_group_closure(n, sym.perm)) {
        if (x.perm.is_identity()) continue;
        const Perm xi = x.perm.inverse();
        bool normal = true;
        for (const SePerm &g : S) {
            Perm c = xi;
            c.permute(g.perm).permute(x.perm);
            bool found = false;
            for (const SePerm &f : S) if (f.perm == c) { found = true; break; }
            if (!found) { normal = false; break; }
        }
        if (normal) h.sym.perm.push_back(x);
    }
    // partition and label rules the symmetrizer leaves unchanged
    bool keep = true;
    for (const SePerm &g : S) keep = keep && allowed_invariant(bis, sym, g.perm);
    if (keep) {
        h.sym.part = sym.part;
        h.sym.label = sym.label;
    }
}

// The launches of one modular contraction (split passes, products,
// recombination) into the arena carena, or, with dd, added to the
// destinations dd names (the caller zeroes their tensor).
void run_crt(ltg_plan *plan, CrtExec *cx, double *carena, int add, const CrtDests *dd) {
    ltg_ctx *ctx = plan->ctx;
    cudaStream_t s = ctx->stream;
    report_device_wait(ctx);
    if (!add && !dd)
        for (auto &r : cx->zero_ranges)
            LTG_CUDA(cudaMemsetAsync(carena + r.first, 0, (r.second - r.first) * sizeof(double), s));
    const double *pa = plan->a->arena.as<double>(), *pb = plan->b->arena.as<double>();
    TimedLaunch t_split(ctx, LTG_KERNEL_OZ_SPLIT);
    LTG_CUDA(launch_crt_fill(cx->nx, cx->ny, cx->ex.as<int32_t>(), cx->ey.as<int32_t>(), s));
    LTG_CUDA(launch_crt_fill(cx->nx, cx->ny, cx->ext.as<int32_t>(), cx->eyt.as<int32_t>(), s));
    LTG_CUDA(launch_crt_fused(plan->fused_split, cx->panels.as<DCrtPanel>(), cx->fams.as<DCrtFamily>(), cx->famp.as<int32_t>(),
                              cx->famt.as<int32_t>(), cx->funits.as<int4>(), cx->nfunits, pa, pb,
                              cx->gidx.as<int32_t>(), cx->ex.as<int32_t>(), cx->ey.as<int32_t>(),
                              cx->res.as<uint8_t>(), cx->cp, s));
    LTG_CUDA(launch_crt_exponents(cx->panels.as<DCrtPanel>(), cx->units.as<int4>(), cx->nunits, cx->nx,
                                  cx->ny, pa, pb, cx->gidx.as<int32_t>(), cx->ex.as<int32_t>(),
                                  cx->ey.as<int32_t>(), cx->sampled, s));
    for (int redo = 0; redo <= cx->sampled; redo++)
        LTG_CUDA(launch_crt_residues(cx->panels.as<DCrtPanel>(), cx->units.as<int4>(), cx->nunits, pa, pb,
                                     cx->gidx.as<int32_t>(), cx->ex.as<int32_t>(), cx->ey.as<int32_t>(),
                                     cx->ext.as<int32_t>(), cx->eyt.as<int32_t>(), cx->sampled, redo,
                                     cx->res.as<uint8_t>(), cx->cp, s));
    t_split.done();
    TimedLaunch t_gemm(ctx, LTG_KERNEL_OZ_GEMM);
    LTG_CUDA(launch_crt_gemm(cx->panels.as<DCrtPanel>(), cx->res.as<uint8_t>(), cx->tasks.as<DCrtTask>(),
                             cx->items.as<DCrtItem>(), cx->cta_items.as<int32_t>(), cx->ncta,
                             cx->out.as<uint8_t>(), cx->cp,
                             ctx->wait_err.as<int32_t>(), ctx->wait_ns, plan->crt_stage_kb, s));
    t_gemm.done();
    TimedLaunch t_comb(ctx, LTG_KERNEL_OZ_COMBINE);
    LTG_CUDA(launch_crt_combine(cx->panels.as<DCrtPanel>(), cx->items.as<DCrtItem>(), cx->nitems,
                                cx->cblks.as<DCBlock>(), cx->comps.as<DCrtComp>(), cx->ctab.as<int32_t>(),
                                cx->cells.as<DCrtCell>(), cx->out.as<uint8_t>(), cx->gidx.as<int32_t>(),
                                cx->ex.as<int32_t>(), cx->ey.as<int32_t>(), cx->ext.as<int32_t>(),
                                cx->eyt.as<int32_t>(), carena, add,
                                cx->scale, cx->cp, s, dd));
    t_comb.done();
    ctx->launches += 4 + (cx->nfunits > 0 ? 1 : 0) + (cx->nunits > 0 ? 2 + cx->sampled : 0) +
                     (cx->nitems > 0 ? 2 : 0);
    fetch_device_wait(ctx);
}

// Sub-dimension groups of one tile axis over the C dims `dims` (in the order
// the axis enumerates them) with extents ext and strides str: unit extents
// dropped, neighbours contiguous in str merged.
SubDims axis_dims(const std::vector<int> &dims, const int64_t *ext, const int64_t *str) {
    SubDims r;
    for (int i : dims) {
        if (ext[i] == 1) continue;
        if (r.n > 0 && r.s0[r.n - 1] == str[i] * ext[i]) {
            r.ext[r.n - 1] *= (int32_t)ext[i];
            r.s0[r.n - 1] = r.s1[r.n - 1] = str[i];
            continue;
        }
        if (r.n == kMaxSub) throw error(kErrUnsupported, "too many sub-dimensions in a symmetrizer term");
        r.ext[r.n] = (int32_t)ext[i];
        r.s0[r.n] = r.s1[r.n] = str[i];
        r.n++;
    }
    return r;
}

// The fused symmetrizer r = c sum_{s in S} sign(s) P_s(T) of the contraction
// T (coefficients ka, kb, kc) in the plain path, for S of two elements.  The
// destinations are the terms of plan_transfer's symmetrizer pass read the
// other way round: result block y and term t read element x_q = y_d, q =
// T.perm[t.perm[d]], of the canonical contraction block behind t^-1(y), so
// that block's element x goes to y with the result block's stride of d on
// its dim q and coefficient c sign(t) (orbit sign).  Each result element has
// one source per term, so it takes at most two atomic adds onto zero, whose
// sum does not depend on their order.
SymExec *prepare_sym(ltg_plan *pl, ltg_bt *r, int32_t mode, int32_t L, double c, int32_t nidx, const int32_t *idx,
                     int32_t symm, double ka, double kb, double kc) {
    const bool crt = mode == LTG_MODE_OZAKI_CRT;
    const bool slice = mode >= LTG_MODE_OZAKI_BF16 && mode <= LTG_MODE_OZAKI_INT8;
    if (mode != LTG_MODE_PLAIN_FP64 && !crt && !slice) throw error(kErrBadArg, "unknown mode");
    if (slice && L != (mode == LTG_MODE_OZAKI_FP8 ? 8 : 7))
        throw error(kErrUnsupported, "the fused symmetrizer in a slice mode takes its default slice count");
    const int n = pl->plan().bisc.n;
    const std::vector<SePerm> S = symmetrizer_group(n, nidx, idx, symm != 0);
    if (S.size() != 2)
        throw error(kErrUnsupported, "the fused symmetrizer takes an index pair or a unitary permutation");
    std::vector<int32_t> skey = {mode, mode != LTG_MODE_PLAIN_FP64 ? L : 0, nidx, symm != 0 ? 1 : 0};
    for (int i = 0; i < (nidx < 0 ? n : nidx); i++) skey.push_back(idx[i]);
    auto key = std::make_tuple(r->uid, skey, c, ka, kb, kc);
    auto it = pl->sym.find(key);
    if (it != pl->sym.end()) return it->second.get();
    if (pl->ctx->capturing) throw error(kErrState, "symmetrizer not prepared before graph capture: call it once outside the capture");
    // the contraction's result space (no arena: its offsets are not used)
    BlockTensorHost th;
    th.bis = pl->plan().bisc;
    th.sym = pl->plan().symc;
    th.build_directory();
    std::vector<GemmTask> tasks;
    std::vector<CBlockTask> cbt;
    contract2_tasks(pl->plan(), pl->a->h, pl->b->h, th, ka, kb, kc, tasks, cbt);
    std::vector<DTask> dt;
    std::vector<DCBlock> dc;
    plain_task_arrays(pl, th.total_elems, tasks, cbt, 1.0, dt, dc);
    // the tile axes: C dims taken from A (m) and from B (n), in C order
    const Contraction &ct = pl->plan().contr;
    const int NC = ct.NC(), NA = ct.NA();
    std::vector<int> mdims, ndims;
    for (int i = 0; i < NC; i++) (ct.conn[i] < NC + NA ? mdims : ndims).push_back(i);
    std::map<int64_t, int32_t> e_of;
    for (size_t e = 0; e < pl->plan().schedule.size(); e++) e_of[pl->plan().schedule[e]] = (int32_t)e;
    const BlockTensorHost &rh = r->h;
    std::unique_ptr<SymExec> ex(new SymExec());
    std::vector<std::vector<DCBlock>> per(cbt.size());
    // the same destinations per dim (result block offset, stride of each
    // contraction dim, coefficient), for the grouped products' cells
    struct DestRec {
        int64_t off;
        int64_t dstr[kMaxOrder];
        double coef;
    };
    std::vector<std::vector<DestRec>> praw(cbt.size());
    int64_t yb[kMaxOrder], xb[kMaxOrder], ext[kMaxOrder], rstr[kMaxOrder], cbi[kMaxOrder], sext[kMaxOrder],
        dstr[kMaxOrder];
    for (size_t sl = 0; sl < rh.blk_abs.size(); sl++) {
        rh.bis.unabs(rh.blk_abs[sl], yb);
        rh.bis.block_dims(yb, ext);
        int64_t st = 1;
        for (int d = n - 1; d >= 0; d--) { rstr[d] = st; st *= ext[d]; }
        bool any = false;
        for (const SePerm &t : S) {
            for (int d = 0; d < n; d++) xb[t.perm.p[d]] = yb[d];
            const int64_t xa = th.bis.abs(xb);
            if (!th.orbits.allowed[xa]) continue;
            const int64_t ca = th.orbits.canon[xa];
            auto f = e_of.find(ca);
            if (f == e_of.end()) continue;                       // a zero block of the contraction
            const int32_t e = f->second;
            if (cbt[e].t_end <= cbt[e].t_begin) continue;
            const Transf &T = th.orbits.tr[xa];
            th.bis.unabs(ca, cbi);
            th.bis.block_dims(cbi, sext);
            for (int d = 0; d < n; d++) {
                const int q = T.perm.p[t.perm.p[d]];
                if (sext[q] != ext[d]) throw error(kErrState, "symmetrizer term extent mismatch");
                dstr[q] = rstr[d];
            }
            DCBlock y;
            std::memset(&y, 0, sizeof(y));
            y.c_off = rh.blk_off[sl];
            // plain: the C block's own scale folded in; modular: the
            // coefficient alone (the recombination applies the global scale)
            y.scale = (crt ? 1.0 : dc[e].scale) * (c * t.coeff * T.coeff);
            y.M = dc[e].M;
            y.N = dc[e].N;
            const SubDims sm = axis_dims(mdims, sext, dstr), sn = axis_dims(ndims, sext, dstr);
            if (sm.total() != y.M || sn.total() != y.N) throw error(kErrState, "symmetrizer term shape");
            pack_sub(sm, y.nm, y.mext, y.mc_str, nullptr);
            pack_sub(sn, y.nn, y.next, y.nc_str, nullptr);
            per[e].push_back(y);
            DestRec q;
            q.off = rh.blk_off[sl];
            for (int d = 0; d < kMaxOrder; d++) q.dstr[d] = d < n ? dstr[d] : 0;
            q.coef = c * t.coeff * T.coeff;
            praw[e].push_back(q);
            any = true;
        }
        if (any) ex->nonzero_slots.push_back((int64_t)sl);
    }
    if (crt) {
        for (size_t e = 0; e < cbt.size(); e++)
            if (per[e].size() > (size_t)kCrtMaxDests)
                throw error(kErrUnsupported, "too many symmetrizer destinations per block for the modular recombination");
        ex->tview.reset(new ltg_bt());
        ex->tview->ctx = pl->ctx;
        ex->tview->h = th;
        ex->crt = prepare_crt(pl, ex->tview.get(), L, ka, kb, kc, 0, 0.0);
    }
    if (slice) {
        ex->tview.reset(new ltg_bt());
        ex->tview->ctx = pl->ctx;
        ex->tview->h = th;
        ex->oz = prepare_ozaki(pl, ex->tview.get(), mode, L, ka, kb, kc, 0, 0.0);
    }
    std::vector<int2> drange(std::max<size_t>(cbt.size(), 1), make_int2(0, 0));
    std::vector<DCBlock> dests;
    for (size_t e = 0; e < cbt.size(); e++) {
        drange[e].x = (int32_t)dests.size();
        dests.insert(dests.end(), per[e].begin(), per[e].end());
        drange[e].y = (int32_t)dests.size();
    }
    ex->ndests = (int64_t)dests.size();
    // small blocks grouped as in the plain path (products into the group
    // buffer; each cell's elements then go to its C block's destinations)
    std::vector<int32_t> group_of(cbt.size(), -1);
    if (!slice && (crt || (pl->group_products && !pl->plan().coalesced))) {
        std::vector<DCrtCell> gcells;
        bool grouped = false;
        if (crt) {
            gcells = ex->crt->cells_host;
            grouped = ex->crt->ngroups > 0;
            if (grouped) {
                std::map<int64_t, int32_t> e_of_off;
                for (size_t e = 0; e < cbt.size(); e++) e_of_off[cbt[e].c_off] = (int32_t)e;
                for (const DCrtCell &cl : gcells) {
                    auto f = e_of_off.find(cl.c_off);
                    if (f != e_of_off.end()) group_of[f->second] = 0;
                }
            }
        } else {
            ex->groups.reset(new PlainGroups());
            build_plain_groups(pl, th, cbt, ka * kb * kc, 1.0, group_of, *ex->groups, &gcells);
            grouped = ex->groups->ngroups > 0;
            if (!grouped) ex->groups.reset();
        }
        if (grouped) {
            std::map<int64_t, int32_t> e_of_off;
            for (size_t e = 0; e < cbt.size(); e++) e_of_off[cbt[e].c_off] = (int32_t)e;
            CrtSideMap sm[2];
            crt_side_maps(ct, th, sm);
            std::vector<int2> gdr(std::max<size_t>(gcells.size(), 1), make_int2(0, 0));
            std::vector<DCrtCell> gdc;
            std::vector<double> gco;
            for (size_t ci = 0; ci < gcells.size(); ci++) {
                auto f = e_of_off.find(gcells[ci].c_off);
                if (f == e_of_off.end() || group_of[f->second] < 0) throw error(kErrState, "grouped cell without its C block");
                gdr[ci].x = (int32_t)gdc.size();
                for (const DestRec &q : praw[f->second]) {
                    DCrtCell d;
                    std::memset(&d, 0, sizeof(d));
                    d.c_off = q.off;
                    for (size_t k = 0; k < sm[0].dims.size(); k++) d.ms[k] = (int32_t)q.dstr[sm[0].dims[k]];
                    for (size_t k = 0; k < sm[1].dims.size(); k++) d.ns[k] = (int32_t)q.dstr[sm[1].dims[k]];
                    gdc.push_back(d);
                    gco.push_back(q.coef);
                }
                gdr[ci].y = (int32_t)gdc.size();
            }
            if (gdc.empty()) { gdc.resize(1); gco.resize(1); }
            cudaStream_t gs = pl->ctx->stream;
            upload_vec(ex->gdrange, gdr, gs);
            upload_vec(ex->gdcells, gdc, gs);
            upload_vec(ex->gdcoef, gco, gs);
        }
    }
    // work items of the other C blocks that reach the result, each over its
    // whole k range (tile shapes as in the plain path)
    std::vector<std::vector<std::pair<double, DItem>>> per_cfg(kNumShapes);
    for (size_t e = 0; e < cbt.size() && !crt && !slice; e++) {
        if (per[e].empty() || group_of[e] >= 0) continue;
        int cfg = pl->forced_tile >= 0 ? pl->forced_tile : pick_tile(cbt[e].M, cbt[e].N);
        auto ov = pl->tile_override.find({cbt[e].M, cbt[e].N});
        if (pl->forced_tile < 0 && ov != pl->tile_override.end()) cfg = ov->second;
        const int bm = tile_cfg_bm(cfg), bn = tile_cfg_bn(cfg);
        for (int64_t m0 = 0; m0 < cbt[e].M; m0 += bm)
            for (int64_t n0 = 0; n0 < cbt[e].N; n0 += bn) {
                DItem di = make_item((int32_t)e, (int32_t)m0, (int32_t)n0);
                const double cost = (double)bm * bn * (cbt[e].kflops + 8.0 * (cbt[e].t_end - cbt[e].t_begin));
                per_cfg[cfg].push_back({cost, di});
            }
    }
    std::vector<DItem> items;
    std::vector<DSplit> splits;
    int64_t ws_elems = 0;
    for (int cfg = 0; cfg < kNumShapes; cfg++)
        append_launch(cfg, per_cfg[cfg], dt, dc, pl->ctx->nsm, 1, items, splits, ws_elems, ex->launches);
    if (!splits.empty()) throw error(kErrState, "k chunks in a fused symmetrizer");
    if (dests.empty()) dests.resize(1);
    cudaStream_t s = pl->ctx->stream;
    upload_vec(ex->tasks, dt, s);
    upload_vec(ex->cblks, dc, s);
    upload_vec(ex->items, items, s);
    upload_vec(ex->drange, drange, s);
    upload_vec(ex->dests, dests, s);
    SymExec *raw = ex.get();
    pl->sym[key] = std::move(ex);
    return raw;
}

}  // namespace

int ltg_bt_create_symmetrized(ltg_bt *a, int32_t nidx, const int32_t *idx, int32_t symm, ltg_bt **out) {
    return guard([&] {
        check_bt(a);
        if (!out) throw error(kErrBadArg, "null output");
        std::unique_ptr<ltg_bt> bt(new ltg_bt());
        bt->ctx = a->ctx;
        symmetrized_space(a->h.bis, a->h.sym, nidx, idx, symm, bt->h);
        alloc_arena(bt.get());
        *out = bt.release();
    });
}

int ltg_symmetrize(ltg_bt *a, double c, int32_t nidx, const int32_t *idx, int32_t symm, ltg_bt *b, int32_t add,
                   double d) {
    return guard([&] {
        check_bt(a);
        check_bt(b);
        need_dev(a->ctx);
        if (!b->h.bis.equals(a->h.bis)) throw error(kErrBadDims, "symmetrizer result of another index space");
        const std::vector<SePerm> S = symmetrizer_group(a->h.bis.n, nidx, idx, symm != 0);
        // passes of at most kMaxTerms_host permuted terms: the first assigns
        // (or adds d times), the others add
        for (size_t t0 = 0; t0 < S.size(); t0 += kMaxTerms_host) {
            std::vector<ltg_bt *> srcs;
            std::vector<Perm> ps;
            std::vector<double> cs;
            for (size_t t = t0; t < std::min(S.size(), t0 + kMaxTerms_host); t++) {
                srcs.push_back(a);
                ps.push_back(S[t].perm);
                cs.push_back(c * S[t].coeff);
            }
            const bool first = t0 == 0;
            run_transfer(a->ctx, srcs, ps, cs, b, first ? add != 0 : true, first ? d : (add ? d : 1.0));
        }
    });
}

int ltg_contract2_make_symmetrized(ltg_plan *plan, int32_t nidx, const int32_t *idx, int32_t symm, ltg_bt **out) {
    return guard([&] {
        if (!plan || !out) throw error(kErrBadArg, "null argument");
        if (plan->external) throw error(kErrUnsupported, "a caller-built task plan has no schedule of its own");
        std::unique_ptr<ltg_bt> bt(new ltg_bt());
        bt->ctx = plan->ctx;
        symmetrized_space(plan->plan().bisc, plan->plan().symc, nidx, idx, symm, bt->h);
        alloc_arena(bt.get());
        *out = bt.release();
    });
}

int ltg_contract2_symmetrized(ltg_plan *plan, ltg_bt *r, int32_t mode, int32_t nslices, double c, int32_t nidx,
                              const int32_t *idx, int32_t symm, double ka, double kb, double kc) {
    return guard([&] {
        if (!plan) throw error(kErrBadArg, "null plan");
        if (plan->external) throw error(kErrUnsupported, "a caller-built task plan has no schedule of its own");
        check_bt(r);
        need_dev(plan->ctx);
        if (!r->h.bis.equals(plan->plan().bisc)) throw error(kErrBadDims, "symmetrizer result of another index space");
        // the result is zeroed before the contraction reads its operands
        if (r == plan->a || r == plan->b)
            throw error(kErrUnsupported, "the fused symmetrizer's result is an operand of the contraction");
        const int L = nslices > 0 ? nslices
                                  : (mode == LTG_MODE_OZAKI_CRT ? 13 : mode == LTG_MODE_OZAKI_FP8 ? 8 : 7);
        SymExec *ex = prepare_sym(plan, r, mode, L, c, nidx, idx, symm, ka, kb, kc);
        ltg_ctx *ctx = plan->ctx;
        cudaStream_t s = ctx->stream;
        // the result starts at zero: every element then takes at most two adds
        LTG_CUDA(cudaMemsetAsync(r->arena.p, 0, (size_t)std::max<int64_t>(r->h.total_elems, 1) * sizeof(double), s));
        if (OzExec *ox = ex->oz) {
            report_device_wait(ctx);
            TimedLaunch t_split(ctx, LTG_KERNEL_OZ_SPLIT);
            LTG_CUDA(launch_oz_split(ox->kind, ox->panels.as<DPanel>(), ox->npanels, ox->max_rows_pad,
                                     plan->a->arena.as<double>(), plan->b->arena.as<double>(),
                                     ox->slices.as<uint8_t>(), ox->exps.as<int32_t>(), ox->S, s));
            t_split.done();
            TimedLaunch t_gemm(ctx, LTG_KERNEL_OZ_GEMM);
            LTG_CUDA(launch_oz_gemm(ox->kind, ox->panels.as<DPanel>(), ox->slices.as<uint8_t>(), ox->tasks.as<DOzTask>(),
                                    ox->cblks.as<DCBlock>(), ox->items.as<DItem>(), ox->nitems,
                                    ox->exps.as<int32_t>(), r->arena.as<double>(), 0, ox->S, ox->chunk_kb,
                                    ctx->wait_err.as<int32_t>(), ctx->wait_ns, s, ex->drange.as<int2>(),
                                    ex->dests.as<DCBlock>()));
            t_gemm.done();
            ctx->launches += 2;
            fetch_device_wait(ctx);
            std::fill(r->h.nonzero.begin(), r->h.nonzero.end(), 0);
            for (int64_t sl : ex->nonzero_slots) r->h.nonzero[sl] = 1;
            return;
        }
        if (ex->crt) {
            const CrtDests dd{ex->drange.as<int2>(), ex->dests.as<DCBlock>(), ex->gdrange.as<int2>(),
                              ex->gdcells.as<DCrtCell>(), ex->gdcoef.as<double>()};
            run_crt(plan, ex->crt, r->arena.as<double>(), 0, &dd);
            std::fill(r->h.nonzero.begin(), r->h.nonzero.end(), 0);
            for (int64_t sl : ex->nonzero_slots) r->h.nonzero[sl] = 1;
            return;
        }
        int slot = 0;
        if (PlainGroups *pg = ex->groups.get()) {
            TimedLaunch tg(ctx, LTG_KERNEL_TRANSFER);
            LTG_CUDA(launch_gather_cells(pg->pieces.as<DGather>(), pg->units.as<int4>(), pg->nunits,
                                         plan->a->arena.as<double>(), plan->b->arena.as<double>(),
                                         pg->buf.as<double>(), s));
            tg.done();
            ctx->launches++;
            for (auto &l : pg->launches) {
                TimedLaunch tl(ctx, LTG_KERNEL_CONTRACT_FP64);
                LTG_CUDA(launch_contract_fp64(pg->tasks.as<DTask>(), pg->cblks.as<DCBlock>(),
                                              pg->items.as<DItem>() + l.item0, l.nitems,
                                              ctx->scratch_counter.as<int32_t>() + (slot++ % 64),
                                              pg->buf.as<double>(), pg->buf.as<double>(), pg->buf.as<double>(),
                                              pg->ws.as<double>() + l.ws_off, 0, l.cfg, s));
                if (l.nsplits > 0) {
                    LTG_CUDA(launch_split_reduce(pg->splits.as<DSplit>() + l.split0, l.nsplits, pg->cblks.as<DCBlock>(),
                                                 pg->ws.as<double>() + l.ws_off, tile_cfg_bm(l.cfg),
                                                 tile_cfg_bn(l.cfg), pg->buf.as<double>(), 0, s));
                    ctx->launches++;
                }
                tl.done();
                ctx->launches++;
            }
            TimedLaunch ts(ctx, LTG_KERNEL_TRANSFER);
            LTG_CUDA(launch_scatter_groups_dest(pg->comps.as<DCrtComp>(), pg->res_off.as<int64_t>(),
                                                pg->ctab.as<int32_t>(), ex->gdrange.as<int2>(),
                                                ex->gdcells.as<DCrtCell>(), ex->gdcoef.as<double>(),
                                                pg->sunits.as<int2>(), pg->nsunits, pg->buf.as<double>(),
                                                r->arena.as<double>(), pg->scale, s));
            ts.done();
            ctx->launches++;
        }
        for (auto &l : ex->launches) {
            TimedLaunch tl(ctx, LTG_KERNEL_CONTRACT_FP64);
            LTG_CUDA(launch_contract_fp64(ex->tasks.as<DTask>(), ex->cblks.as<DCBlock>(),
                                          ex->items.as<DItem>() + l.item0, l.nitems,
                                          ctx->scratch_counter.as<int32_t>() + (slot++ % 64),
                                          plan->a->arena.as<double>(), plan->b->arena.as<double>(),
                                          r->arena.as<double>(), nullptr, 0, l.cfg, s, ex->drange.as<int2>(),
                                          ex->dests.as<DCBlock>()));
            tl.done();
            ctx->launches++;
        }
        std::fill(r->h.nonzero.begin(), r->h.nonzero.end(), 0);
        for (int64_t sl : ex->nonzero_slots) r->h.nonzero[sl] = 1;
        if (!ctx->capturing) LTG_CUDA(cudaGetLastError());
    });
}

int ltg_bt_destroy(ltg_bt *bt) {
    return guard([&] {
        check_bt(bt);
        forget_dot(bt);
        forget_transfer(bt);
        if (bt->ctx->device >= 0) cudaStreamSynchronize(bt->ctx->stream);
        delete bt;
    });
}

int ltg_bt_info(const ltg_bt *bt, int32_t *order, int64_t *nblocks, int64_t *nelems) {
    return guard([&] {
        check_bt(bt);
        if (order) *order = bt->h.bis.n;
        if (nblocks) *nblocks = (int64_t)bt->h.blk_abs.size();
        if (nelems) *nelems = bt->h.total_elems;
    });
}

int ltg_bt_blocks(const ltg_bt *bt, int64_t *abs_idx, int64_t *offset, int64_t *size) {
    return guard([&] {
        check_bt(bt);
        for (size_t i = 0; i < bt->h.blk_abs.size(); i++) {
            if (abs_idx) abs_idx[i] = bt->h.blk_abs[i];
            if (offset) offset[i] = bt->h.blk_off[i];
            if (size) size[i] = bt->h.blk_size[i];
        }
    });
}

int ltg_bt_bidims(const ltg_bt *bt, int64_t *bidims) {
    return guard([&] {
        check_bt(bt);
        for (int d = 0; d < bt->h.bis.n; d++) bidims[d] = bt->h.bis.bidims[d];
    });
}

int ltg_bt_block_dims(const ltg_bt *bt, const int64_t *bidx, int64_t *dims) {
    return guard([&] {
        check_bt(bt);
        if (!bidx || !dims) throw error(kErrBadArg, "null argument");
        for (int d = 0; d < bt->h.bis.n; d++)
            if (bidx[d] < 0 || bidx[d] >= bt->h.bis.bidims[d]) throw error(kErrBadArg, "block index out of range");
        bt->h.bis.block_dims(bidx, dims);
    });
}

int ltg_bt_nonzero(const ltg_bt *bt, int64_t *abs_idx, int64_t cap, int64_t *n) {
    return guard([&] {
        check_bt(bt);
        int64_t k = 0;
        for (size_t i = 0; i < bt->h.blk_abs.size(); i++) {
            if (!bt->h.nonzero[i]) continue;
            if (abs_idx && k < cap) abs_idx[k] = bt->h.blk_abs[i];
            k++;
        }
        if (n) *n = k;
    });
}

int ltg_bt_orbit(const ltg_bt *bt, int64_t abs_idx, int64_t *canonical, int32_t *perm,
                 double *coeff, int32_t *allowed) {
    return guard([&] {
        check_bt(bt);
        if (abs_idx < 0 || abs_idx >= bt->h.bis.nblocks()) throw error(kErrBadArg, "block index out of range");
        const OrbitTable &o = bt->h.orbits;
        if (canonical) *canonical = o.canon[abs_idx];
        if (perm) for (int d = 0; d < bt->h.bis.n; d++) perm[d] = o.tr[abs_idx].perm.n ? o.tr[abs_idx].perm.p[d] : d;
        if (coeff) *coeff = o.tr[abs_idx].coeff;
        if (allowed) *allowed = o.allowed[abs_idx];
    });
}

int ltg_bt_upload(ltg_bt *bt, const double *host) {
    return guard([&] {
        check_bt(bt);
        need_dev(bt->ctx);
        if (!host) throw error(kErrBadArg, "null host buffer");
        LTG_CUDA(cudaMemcpyAsync(bt->arena.p, host, bt->h.total_elems * sizeof(double), cudaMemcpyHostToDevice, bt->ctx->stream));
        LTG_CUDA(cudaStreamSynchronize(bt->ctx->stream));
        std::fill(bt->h.nonzero.begin(), bt->h.nonzero.end(), 1);
    });
}

int ltg_bt_download(ltg_bt *bt, double *host) {
    return guard([&] {
        check_bt(bt);
        need_dev(bt->ctx);
        if (!host) throw error(kErrBadArg, "null host buffer");
        LTG_CUDA(cudaMemcpyAsync(host, bt->arena.p, bt->h.total_elems * sizeof(double), cudaMemcpyDeviceToHost, bt->ctx->stream));
        LTG_CUDA(cudaStreamSynchronize(bt->ctx->stream));
    });
}

int ltg_bt_upload_async(ltg_bt *bt, const double *host) {
    return guard([&] {
        check_bt(bt);
        need_dev(bt->ctx);
        if (!host) throw error(kErrBadArg, "null host buffer");
        LTG_CUDA(cudaMemcpyAsync(bt->arena.p, host, bt->h.total_elems * sizeof(double), cudaMemcpyHostToDevice, bt->ctx->stream));
        std::fill(bt->h.nonzero.begin(), bt->h.nonzero.end(), 1);
    });
}

int ltg_bt_download_async(ltg_bt *bt, double *host) {
    return guard([&] {
        check_bt(bt);
        need_dev(bt->ctx);
        if (!host) throw error(kErrBadArg, "null host buffer");
        LTG_CUDA(cudaMemcpyAsync(host, bt->arena.p, bt->h.total_elems * sizeof(double), cudaMemcpyDeviceToHost, bt->ctx->stream));
    });
}

static int64_t slot_of_bidx(const ltg_bt *bt, const int64_t *bidx) {
    for (int d = 0; d < bt->h.bis.n; d++)
        if (bidx[d] < 0 || bidx[d] >= bt->h.bis.bidims[d]) throw error(kErrBadArg, "block index out of range");
    int64_t a = bt->h.bis.abs(bidx);
    int64_t s = bt->h.slot_of[a];
    if (s < 0) throw error(kErrSymmetry, "block is not canonical or not allowed by the symmetry");
    return s;
}

int ltg_bt_upload_block(ltg_bt *bt, const int64_t *bidx, const double *data) {
    return guard([&] {
        check_bt(bt);
        need_dev(bt->ctx);
        int64_t s = slot_of_bidx(bt, bidx);
        LTG_CUDA(cudaMemcpyAsync(bt->arena.as<double>() + bt->h.blk_off[s], data, bt->h.blk_size[s] * sizeof(double), cudaMemcpyHostToDevice, bt->ctx->stream));
        LTG_CUDA(cudaStreamSynchronize(bt->ctx->stream));
        bt->h.nonzero[s] = 1;
    });
}

int ltg_bt_download_block(ltg_bt *bt, const int64_t *bidx, double *data) {
    return guard([&] {
        check_bt(bt);
        need_dev(bt->ctx);
        int64_t s = slot_of_bidx(bt, bidx);
        LTG_CUDA(cudaMemcpyAsync(data, bt->arena.as<double>() + bt->h.blk_off[s], bt->h.blk_size[s] * sizeof(double), cudaMemcpyDeviceToHost, bt->ctx->stream));
        LTG_CUDA(cudaStreamSynchronize(bt->ctx->stream));
    });
}

int ltg_bt_set_zero(ltg_bt *bt) {
    return guard([&] {
        check_bt(bt);
        need_dev(bt->ctx);
        LTG_CUDA(cudaMemsetAsync(bt->arena.p, 0, std::max<int64_t>(bt->h.total_elems, 1) * sizeof(double), bt->ctx->stream));
        std::fill(bt->h.nonzero.begin(), bt->h.nonzero.end(), 0);
    });
}

int ltg_bt_zero_block(ltg_bt *bt, const int64_t *bidx) {
    return guard([&] {
        check_bt(bt);
        int64_t s = slot_of_bidx(bt, bidx);
        if (bt->ctx->device >= 0)
            LTG_CUDA(cudaMemsetAsync(bt->arena.as<double>() + bt->h.blk_off[s], 0,
                                     bt->h.blk_size[s] * sizeof(double), bt->ctx->stream));
        bt->h.nonzero[s] = 0;
    });
}

int ltg_bt_mark_nonzero(ltg_bt *bt) {
    return guard([&] { check_bt(bt); std::fill(bt->h.nonzero.begin(), bt->h.nonzero.end(), 1); });
}

int ltg_bt_fill_seeded(ltg_bt *bt, uint64_t seed, double scale) {
    return guard([&] {
        check_bt(bt);
        need_dev(bt->ctx);
        upload_directory(bt);
        DGenGroup g = gen_group(bt->h);
        TimedLaunch tl(bt->ctx, LTG_KERNEL_FILL);
        LTG_CUDA(launch_fill_seeded(bt->arena.as<double>(), bt->dir_off.as<int64_t>(), bt->dir_start.as<int64_t>(),
                                    bt->dir_ext.as<int32_t>(), (int32_t)bt->h.blk_abs.size(), bt->h.bis.n, g, seed,
                                    two_m32(scale), bt->ctx->stream));
        tl.done();
        bt->ctx->launches++;
        LTG_CUDA(cudaStreamSynchronize(bt->ctx->stream));
        std::fill(bt->h.nonzero.begin(), bt->h.nonzero.end(), 1);
    });
}

int ltg_bt_fill_seeded_host(const ltg_bt *bt, uint64_t seed, double scale, double *host) {
    return guard([&] {
        check_bt(bt);
        if (!host) throw error(kErrBadArg, "null host buffer");
        DGenGroup g = gen_group(bt->h);
        const BlockTensorHost &h = bt->h;
        const double sc = two_m32(scale);
        int nt = std::max(1, std::min(bt->ctx->host_threads, 64));
        std::vector<std::thread> th;
        for (int w = 0; w < nt; w++) {
            th.emplace_back([&, w] {
                int64_t bidx[kMaxOrder], ext[kMaxOrder], x[kMaxOrder];
                for (size_t i = w; i < h.blk_abs.size(); i += nt) {
                    h.bis.unabs(h.blk_abs[i], bidx);
                    h.bis.block_dims(bidx, ext);
                    double *dst = host + h.blk_off[i];
                    for (int64_t e = 0; e < h.blk_size[i]; e++) {
                        int64_t r = e;
                        for (int d = h.bis.n - 1; d >= 0; d--) {
                            x[d] = h.bis.starts[d][bidx[d]] + r % ext[d];
                            r /= ext[d];
                        }
                        dst[e] = seeded_value(g, seed, sc, x);
                    }
                    for (int64_t e = h.blk_size[i]; e < ((h.blk_size[i] + 3) & ~int64_t(3)); e++)
                        if (h.blk_off[i] + e < h.total_elems) dst[e] = 0.0;
                }
            });
        }
        for (auto &t : th) t.join();
    });
}

int ltg_bt_device_ptr(ltg_bt *bt, double **ptr) {
    return guard([&] { check_bt(bt); if (!ptr) throw error(kErrBadArg, "null output"); *ptr = bt->arena.as<double>(); });
}

namespace {
// Process-wide cache of contraction schedules.  The schedule (non-zero C
// blocks, coalesced pair lists, result space) depends only on the
// contraction and on both operands' block index spaces, symmetries and
// non-zero block sets, so operations built again from tensors of the same
// description -- every iteration of a coupled-cluster program, every
// letter-interface assignment -- reuse it.  Keyed by all of that, least
// recently used entries dropped beyond the capacity.
struct ScheduleCache {
    std::mutex mtx;
    std::list<std::pair<std::string, std::shared_ptr<const ContractPlan>>> lru;   // most recent first
    std::map<std::string, decltype(lru)::iterator> index;
    size_t capacity = 64;
    int64_t hits = 0, misses = 0;
};
ScheduleCache &schedule_cache() {
    static ScheduleCache c;
    return c;
}

void key_put(std::string &k, int64_t v) { k.append(reinterpret_cast<const char *>(&v), sizeof(v)); }
void key_putd(std::string &k, double v) { k.append(reinterpret_cast<const char *>(&v), sizeof(v)); }

void key_tensor(std::string &k, const BlockTensorHost &h) {
    const Bis &b = h.bis;
    key_put(k, (int64_t)b.n);
    for (int d = 0; d < b.n; d++) {
        key_put(k, b.dims[d]);
        key_put(k, (int64_t)b.starts[d].size());
        for (int64_t x : b.starts[d]) key_put(k, x);
    }
    key_put(k, (int64_t)h.sym.perm.size());
    for (const SePerm &e : h.sym.perm) {
        for (int d = 0; d < b.n; d++) key_put(k, (int64_t)e.perm.p[d]);
        key_putd(k, e.coeff);
    }
    key_put(k, (int64_t)h.sym.part.size());
    for (const SePart &q : h.sym.part) {
        for (int d = 0; d < b.n; d++) { key_put(k, q.pdims[d]); key_put(k, q.bipdims[d]); }
        key_put(k, (int64_t)q.forbidden.size());
        k.append(q.forbidden.begin(), q.forbidden.end());
    }
    key_put(k, (int64_t)h.sym.label.size());
    for (const SeLabel &l : h.sym.label) {
        key_put(k, (int64_t)l.nirrep);
        for (int d = 0; d < b.n; d++) {
            key_put(k, (int64_t)l.labels[d].size());
            for (int x : l.labels[d]) key_put(k, (int64_t)x);
        }
        key_put(k, (int64_t)l.rule.size());
        for (const auto &prod : l.rule) {
            key_put(k, (int64_t)prod.size());
            for (const LabelTerm &t : prod) {
                for (int d = 0; d < b.n; d++) key_put(k, (int64_t)t.seq[d]);
                key_put(k, (int64_t)t.intr);
            }
        }
    }
    key_put(k, (int64_t)h.nonzero.size());
    k.append(h.nonzero.begin(), h.nonzero.end());
}
}  // namespace

int ltg_schedule_cache_set_capacity(int64_t entries) {
    return guard([&] {
        if (entries < 0) throw error(kErrBadArg, "negative capacity");
        ScheduleCache &c = schedule_cache();
        std::lock_guard<std::mutex> lk(c.mtx);
        c.capacity = (size_t)entries;
        while (c.lru.size() > c.capacity) {
            c.index.erase(c.lru.back().first);
            c.lru.pop_back();
        }
    });
}

int ltg_schedule_cache_stats(int64_t *hits, int64_t *misses, int64_t *entries) {
    return guard([&] {
        ScheduleCache &c = schedule_cache();
        std::lock_guard<std::mutex> lk(c.mtx);
        if (hits) *hits = c.hits;
        if (misses) *misses = c.misses;
        if (entries) *entries = (int64_t)c.lru.size();
    });
}

int ltg_contract2_create(ltg_ctx *ctx, int32_t n, int32_t m, int32_t k, const int32_t *permc,
                         const int32_t *pairs, ltg_bt *a, ltg_bt *b, ltg_plan **out) {
    return guard([&] {
        check_ctx(ctx); check_bt(a); check_bt(b);
        if (!out) throw error(kErrBadArg, "null output");
        if (n < 0 || m < 0 || k < 0 || n + m < 1) throw error(kErrBadArg, "invalid contraction orders");
        if (a->h.bis.n != n + k || b->h.bis.n != m + k) throw error(kErrBadDims, "argument orders do not match the contraction");
        std::unique_ptr<ltg_plan> pl(new ltg_plan());
        pl->ctx = ctx; pl->a = a; pl->b = b;
        Contraction c;
        c.init(n, m, k, perm_from(n + m, permc));
        for (int q = 0; q < k; q++) c.contract(pairs[2 * q], pairs[2 * q + 1]);
        std::string key;
        key_put(key, (int64_t)n); key_put(key, (int64_t)m); key_put(key, (int64_t)k);
        const Perm pc = perm_from(n + m, permc);
        for (int d = 0; d < n + m; d++) key_put(key, (int64_t)pc.p[d]);
        for (int q = 0; q < 2 * k; q++) key_put(key, (int64_t)pairs[q]);
        key_tensor(key, a->h);
        key_tensor(key, b->h);
        ScheduleCache &sc = schedule_cache();
        {
            std::lock_guard<std::mutex> lk(sc.mtx);
            auto f = sc.index.find(key);
            if (f != sc.index.end()) {
                sc.lru.splice(sc.lru.begin(), sc.lru, f->second);
                pl->planp = f->second->second;
                sc.hits++;
                *out = pl.release();
                return;
            }
            sc.misses++;
        }
        std::shared_ptr<ContractPlan> cp = std::make_shared<ContractPlan>();
        contract2_schedule(c, a->h, b->h, *cp, ctx->host_threads);
        pl->planp = cp;
        {
            std::lock_guard<std::mutex> lk(sc.mtx);
            if (sc.capacity > 0 && sc.index.find(key) == sc.index.end()) {
                sc.lru.emplace_front(key, pl->planp);
                sc.index[key] = sc.lru.begin();
                while (sc.lru.size() > sc.capacity) {
                    sc.index.erase(sc.lru.back().first);
                    sc.lru.pop_back();
                }
            }
        }
        *out = pl.release();
    });
}

int ltg_contract2_make_result(ltg_plan *plan, ltg_bt **c) {
    return guard([&] {
        if (!plan || !c) throw error(kErrBadArg, "null argument");
        if (plan->external) throw error(kErrUnsupported, "a caller-built task plan has no schedule of its own");
        std::unique_ptr<ltg_bt> bt(new ltg_bt());
        bt->ctx = plan->ctx;
        bt->h.bis = plan->plan().bisc;
        bt->h.sym = plan->plan().symc;
        alloc_arena(bt.get());
        *c = bt.release();
    });
}

int ltg_plan_schedule(ltg_plan *plan, int64_t *abs_idx, int64_t cap, int64_t *n) {
    return guard([&] {
        if (!plan) throw error(kErrBadArg, "null plan");
        const auto &s = plan->plan().schedule;
        for (size_t i = 0; i < s.size() && (int64_t)i < cap; i++) abs_idx[i] = s[i];
        if (n) *n = (int64_t)s.size();
    });
}

int ltg_plan_pairs(ltg_plan *plan, int64_t i, int64_t *out, int64_t cap, int64_t *npairs) {
    return guard([&] {
        if (!plan) throw error(kErrBadArg, "null plan");
        if (i < 0 || i >= (int64_t)plan->plan().clst.size()) throw error(kErrBadArg, "schedule index out of range");
        const auto &lst = plan->plan().clst[i];
        const int NA = plan->plan().contr.NA(), NB = plan->plan().contr.NB();
        const int64_t rec = 2 + NA + 1 + 2 + NB + 1;
        int64_t k = 0;
        for (const Pair &p : lst) {
            if ((k + 1) * rec <= cap) {
                int64_t *o = out + k * rec;
                o[0] = p.aia; o[1] = p.acia;
                for (int d = 0; d < NA; d++) o[2 + d] = p.tra.perm.n ? p.tra.perm.p[d] : d;
                std::memcpy(&o[2 + NA], &p.tra.coeff, 8);
                int64_t *q = o + 3 + NA;
                q[0] = p.aib; q[1] = p.acib;
                for (int d = 0; d < NB; d++) q[2 + d] = p.trb.perm.n ? p.trb.perm.p[d] : d;
                std::memcpy(&q[2 + NB], &p.trb.coeff, 8);
            }
            k++;
        }
        if (npairs) *npairs = k;
    });
}

int ltg_plan_flops(ltg_plan *plan, double *flops) {
    return guard([&] { if (!plan || !flops) throw error(kErrBadArg, "null argument"); *flops = plan->plan().flops; });
}



int ltg_plan_export_tasks(ltg_plan *plan, ltg_bt *c, int64_t *tasks, int64_t cap, int64_t *ntasks) {
    return guard([&] {
        if (!plan || !ntasks) throw error(kErrBadArg, "null argument");
        check_bt(c);
        if (plan->external) throw error(kErrBadArg, "the plan holds caller-built tasks");
        if (!c->h.bis.equals(plan->plan().bisc)) throw error(kErrBadDims, "result tensor has a different block index space");
        std::vector<GemmTask> t;
        std::vector<CBlockTask> cbt;
        contract2_tasks(plan->plan(), plan->a->h, plan->b->h, c->h, 1.0, 1.0, 1.0, t, cbt);
        for (size_t i = 0; i < t.size() && (int64_t)i < cap; i++) pack_task(t[i], tasks + LTG_TASK_WORDS * i);
        *ntasks = (int64_t)t.size();
    });
}

int ltg_plan_contract2_upload(ltg_ctx *ctx, ltg_bt *a, ltg_bt *b, const int64_t *tasks, int64_t ntasks,
                              ltg_plan **out) {
    return guard([&] {
        check_ctx(ctx); check_bt(a); check_bt(b);
        if (!out || (ntasks > 0 && !tasks) || ntasks < 0) throw error(kErrBadArg, "invalid task list");
        std::unique_ptr<ltg_plan> pl(new ltg_plan());
        pl->ctx = ctx; pl->a = a; pl->b = b;
        pl->external = true;
        std::shared_ptr<ContractPlan> cp = std::make_shared<ContractPlan>();
        cp->coalesced = true;
        for (int64_t i = 0; i < ntasks; i++) {
            pl->ext_tasks.push_back(unpack_task(tasks + LTG_TASK_WORDS * i));
            const GemmTask &t = pl->ext_tasks.back();
            cp->flops += 2.0 * (double)t.m.total() * (double)t.n.total() * (double)t.k.total();
        }
        pl->planp = cp;
        *out = pl.release();
    });
}

// Names of the boundary as first specified (aliases of the entry points above).
int ltg_bt_alloc(ltg_ctx *ctx, const ltg_bt_spec *spec, ltg_bt **out) { return ltg_bt_create(ctx, spec, out); }
int ltg_bt_free(ltg_bt *bt) { return ltg_bt_destroy(bt); }
int ltg_bt_upload_blocks(ltg_bt *bt, const double *host) { return ltg_bt_upload(bt, host); }
int ltg_bt_download_blocks(ltg_bt *bt, double *host) { return ltg_bt_download(bt, host); }
int ltg_plan_free(ltg_plan *plan) { return ltg_plan_destroy(plan); }
int ltg_copy_perm(ltg_bt *a, const int32_t *perm, double c, ltg_bt *b, int32_t add, double d) {
    return ltg_copy(a, perm, c, b, add, d);
}
int ltg_add_perm_n(int32_t nterms, ltg_bt *const *a, const int32_t *perms, const double *coeffs, ltg_bt *b,
                   int32_t add, double d) {
    return ltg_add(nterms, a, perms, coeffs, b, add, d);
}
const char *ltg_last_error_string(void) { return ltg_last_error(); }

int ltg_contract2(ltg_plan *plan, ltg_bt *c, int32_t mode, int32_t nslices, double ka, double kb,
                  double kc, int32_t add, double d) {
    return guard([&] {
        if (!plan) throw error(kErrBadArg, "null plan");
        check_bt(c);
        need_dev(plan->ctx);
        if (plan->external) {
            if (mode != LTG_MODE_PLAIN_FP64) throw error(kErrUnsupported, "a caller-built task plan runs in the plain FP64 mode only");
        } else if (!c->h.bis.equals(plan->plan().bisc)) {
            throw error(kErrBadDims, "result tensor has a different block index space");
        }
        ltg_ctx *ctx = plan->ctx;
        cudaStream_t s = ctx->stream;
        if (mode == LTG_MODE_OZAKI_CRT) {
            CrtExec *cx = prepare_crt(plan, c, nslices > 0 ? nslices : 13, ka, kb, kc, add, d);
            run_crt(plan, cx, c->arena.as<double>(), add, nullptr);
            if (!add) std::fill(c->h.nonzero.begin(), c->h.nonzero.end(), 0);
            for (int64_t sl : cx->sched_slots) c->h.nonzero[sl] = 1;
            return;
        }
        if (mode != LTG_MODE_PLAIN_FP64) {
            if (mode < LTG_MODE_OZAKI_BF16 || mode > LTG_MODE_OZAKI_INT8) throw error(kErrBadArg, "unknown mode");
            int S = nslices > 0 ? nslices : (mode == LTG_MODE_OZAKI_FP8 ? 8 : 7);
            OzExec *ox = prepare_ozaki(plan, c, mode, S, ka, kb, kc, add, d);
            report_device_wait(ctx);
            if (!add)
                for (auto &r : ox->zero_ranges)
                    LTG_CUDA(cudaMemsetAsync(c->arena.as<double>() + r.first, 0, (r.second - r.first) * sizeof(double), s));
            TimedLaunch t_split(ctx, LTG_KERNEL_OZ_SPLIT);
            LTG_CUDA(launch_oz_split(ox->kind, ox->panels.as<DPanel>(), ox->npanels, ox->max_rows_pad,
                                     plan->a->arena.as<double>(), plan->b->arena.as<double>(),
                                     ox->slices.as<uint8_t>(), ox->exps.as<int32_t>(), ox->S, s));
            t_split.done();
            TimedLaunch t_gemm(ctx, LTG_KERNEL_OZ_GEMM);
            LTG_CUDA(launch_oz_gemm(ox->kind, ox->panels.as<DPanel>(), ox->slices.as<uint8_t>(), ox->tasks.as<DOzTask>(),
                                    ox->cblks.as<DCBlock>(), ox->items.as<DItem>(), ox->nitems,
                                    ox->exps.as<int32_t>(), c->arena.as<double>(), add, ox->S, ox->chunk_kb,
                                    ctx->wait_err.as<int32_t>(), ctx->wait_ns, s));
            t_gemm.done();
            ctx->launches += 2;
            fetch_device_wait(ctx);
            if (!add) std::fill(c->h.nonzero.begin(), c->h.nonzero.end(), 0);
            for (int64_t sl : ox->sched_slots) c->h.nonzero[sl] = 1;
            return;
        }
        ContractExec *ex = prepare_exec(plan, c, ka, kb, kc, add, d);
        if (!add)
            for (auto &r : ex->zero_ranges)
                LTG_CUDA(cudaMemsetAsync(c->arena.as<double>() + r.first, 0, (r.second - r.first) * sizeof(double), s));
        int slot = 0;
        PlainGroups *pg = ex->groups.get();
        if (pg) {
            TimedLaunch tg(ctx, LTG_KERNEL_TRANSFER);
            LTG_CUDA(launch_gather_cells(pg->pieces.as<DGather>(), pg->units.as<int4>(), pg->nunits,
                                         plan->a->arena.as<double>(), plan->b->arena.as<double>(),
                                         pg->buf.as<double>(), s));
            tg.done();
            ctx->launches++;
            for (auto &l : pg->launches) {
                TimedLaunch tl(ctx, LTG_KERNEL_CONTRACT_FP64);
                LTG_CUDA(launch_contract_fp64(pg->tasks.as<DTask>(), pg->cblks.as<DCBlock>(),
                                              pg->items.as<DItem>() + l.item0, l.nitems,
                                              ctx->scratch_counter.as<int32_t>() + (slot++ % 64),
                                              pg->buf.as<double>(), pg->buf.as<double>(), pg->buf.as<double>(),
                                              pg->ws.as<double>() + l.ws_off, 0, l.cfg, s));
                if (l.nsplits > 0) {
                    LTG_CUDA(launch_split_reduce(pg->splits.as<DSplit>() + l.split0, l.nsplits, pg->cblks.as<DCBlock>(),
                                                 pg->ws.as<double>() + l.ws_off, tile_cfg_bm(l.cfg),
                                                 tile_cfg_bn(l.cfg), pg->buf.as<double>(), 0, s));
                    ctx->launches++;
                }
                tl.done();
                ctx->launches++;
            }
        }
        for (auto &l : ex->launches) {
            TimedLaunch tl(ctx, LTG_KERNEL_CONTRACT_FP64);
            LTG_CUDA(launch_contract_fp64(ex->tasks.as<DTask>(), ex->cblks.as<DCBlock>(),
                                          ex->items.as<DItem>() + l.item0, l.nitems,
                                          ctx->scratch_counter.as<int32_t>() + (slot++ % 64),
                                          plan->a->arena.as<double>(), plan->b->arena.as<double>(),
                                          c->arena.as<double>(), ex->ws.as<double>() + l.ws_off, add, l.cfg, s));
            if (l.nsplits > 0) {
                LTG_CUDA(launch_split_reduce(ex->splits.as<DSplit>() + l.split0, l.nsplits, ex->cblks.as<DCBlock>(),
                                             ex->ws.as<double>() + l.ws_off, tile_cfg_bm(l.cfg), tile_cfg_bn(l.cfg),
                                             c->arena.as<double>(), add, s));
                ctx->launches++;
            }
            tl.done();
            ctx->launches++;
        }
        if (pg) {
            TimedLaunch ts(ctx, LTG_KERNEL_TRANSFER);
            LTG_CUDA(launch_scatter_groups(pg->comps.as<DCrtComp>(), pg->res_off.as<int64_t>(), pg->ctab.as<int32_t>(),
                                           pg->cells.as<DCrtCell>(), pg->sunits.as<int2>(), pg->nsunits,
                                           pg->buf.as<double>(), c->arena.as<double>(), pg->scale, add, s));
            ts.done();
            ctx->launches++;
        }
        if (!add) std::fill(c->h.nonzero.begin(), c->h.nonzero.end(), 0);
        for (int64_t sl : ex->sched_slots) c->h.nonzero[sl] = 1;
        if (!ctx->capturing) LTG_CUDA(cudaGetLastError());
    });
}

int ltg_contract2_split_bytes(ltg_plan *plan, ltg_bt *c, int32_t mode, int32_t nslices, double ka, double kb,
                              double kc, int32_t add, double d, int64_t *read_bytes, int64_t *write_bytes) {
    return guard([&] {
        if (!plan || !read_bytes || !write_bytes) throw error(kErrBadArg, "null argument");
        if (plan->external) throw error(kErrUnsupported, "a caller-built task plan has no schedule of its own");
        check_bt(c);
        need_dev(plan->ctx);
        if (mode == LTG_MODE_OZAKI_CRT) {
            CrtExec *cx = prepare_crt(plan, c, nslices > 0 ? nslices : 13, ka, kb, kc, add, d);
            // row families: one HBM read (the second pass reads L2); the other
            // panels: the exponent pass and the residue pass
            *read_bytes = 8 * (cx->exp_elems + cx->src_elems);
            *write_bytes = cx->res_bytes;
        } else if (mode >= LTG_MODE_OZAKI_BF16 && mode <= LTG_MODE_OZAKI_INT8) {
            const int S = nslices > 0 ? nslices : (mode == LTG_MODE_OZAKI_FP8 ? 8 : 7);
            OzExec *ox = prepare_ozaki(plan, c, mode, S, ka, kb, kc, add, d);
            *read_bytes = 8 * ox->src_elems;
            *write_bytes = ox->slice_bytes;
        } else {
            throw error(kErrBadArg, "not a split-precision mode");
        }
    });
}

int ltg_plan_destroy(ltg_plan *plan) {
    return guard([&] {
        if (!plan) throw error(kErrBadArg, "null plan");
        if (plan->ctx->device >= 0) cudaStreamSynchronize(plan->ctx->stream);
        delete plan;
    });
}

int ltg_contract2_set_tile(ltg_plan *plan, int32_t cfg) {
    return guard([&] {
        if (!plan) throw error(kErrBadArg, "null plan");
        if (cfg < -1 || cfg >= tile_cfg_count()) throw error(kErrBadArg, "tile configuration out of range");
        plan->forced_tile = cfg;
        plan->exec.clear();
        plan->sym.clear();
    });
}

int ltg_contract2_set_split_k(ltg_plan *plan, int32_t k) {
    return guard([&] {
        if (!plan) throw error(kErrBadArg, "null plan");
        if (k < 0 || k > 4) throw error(kErrBadArg, "k chunks per tile must be 0 (automatic) or 1-4");
        plan->split_k = k;
        plan->exec.clear();
        plan->sym.clear();
    });
}

int ltg_contract2_set_grouping(ltg_plan *plan, int32_t enable) {
    return guard([&] {
        if (!plan) throw error(kErrBadArg, "null plan");
        if (plan->ctx->capturing) throw error(kErrState, "cannot change a plan during graph capture");
        plan->group_products = enable != 0;
        plan->crt.clear();
        plan->sym.clear();              // modular symmetrizers point into plan->crt
    });
}

int ltg_contract2_set_fused_split(ltg_plan *plan, int32_t enable) {
    return guard([&] {
        if (!plan) throw error(kErrBadArg, "null plan");
        if (plan->ctx->capturing) throw error(kErrState, "cannot change a plan during graph capture");
        if (enable < 0 || enable > 2) throw error(kErrBadArg, "one-read split shape must be 0 (off), 1 or 2");
        plan->fused_split = enable;
        plan->crt.clear();
        plan->sym.clear();              // modular symmetrizers point into plan->crt
    });
}

int ltg_contract2_set_crt_bound(ltg_plan *plan, int32_t sampled) {
    return guard([&] {
        if (!plan) throw error(kErrBadArg, "null plan");
        if (plan->ctx->capturing) throw error(kErrState, "cannot change a plan during graph capture");
        if (sampled != 0 && sampled != 1) throw error(kErrBadArg, "exponent bound must be 0 (exact) or 1 (sampled)");
        plan->crt_sampled = sampled;
        plan->crt.clear();
        plan->sym.clear();              // modular symmetrizers point into plan->crt
    });
}

int ltg_contract2_set_crt_stage(ltg_plan *plan, int32_t kblocks) {
    return guard([&] {
        if (!plan) throw error(kErrBadArg, "null plan");
        if (kblocks != 2 && kblocks != 3 && kblocks != 4 && kblocks != 6)
            throw error(kErrBadArg, "k blocks per stage must be 2, 3, 4 or 6");
        plan->crt_stage_kb = kblocks;
    });
}

int ltg_contract2_set_crt_rows(ltg_plan *plan, int32_t rows) {
    return guard([&] {
        if (!plan) throw error(kErrBadArg, "null plan");
        if (rows != 0 && rows != 128 && rows != 256) throw error(kErrBadArg, "work-item rows must be 0, 128 or 256");
        if (plan->ctx->capturing) throw error(kErrState, "cannot change a plan during graph capture");
        plan->crt_rows = rows;
        plan->crt.clear();
        plan->sym.clear();              // modular symmetrizers point into plan->crt
    });
}

int ltg_contract2_group_info(ltg_plan *plan, ltg_bt *c, int64_t *ngroups, int64_t *nblocks,
                             double *grouped_flops, double *block_flops) {
    return guard([&] {
        if (!plan) throw error(kErrBadArg, "null plan");
        if (plan->external) throw error(kErrUnsupported, "a caller-built task plan has no schedule of its own");
        check_bt(c);
        if (!c->h.bis.equals(plan->plan().bisc)) throw error(kErrBadDims, "result tensor has a different block index space");
        std::vector<GemmTask> tasks;
        std::vector<CBlockTask> cbt;
        contract2_tasks(plan->plan(), plan->a->h, plan->b->h, c->h, 1.0, 1.0, 1.0, tasks, cbt);
        CrtSideMap sm[2];
        crt_side_maps(plan->plan().contr, c->h, sm);
        std::vector<CrtGroupHost> groups;
        std::vector<int32_t> group_of(cbt.size(), -1);
        if (plan->group_products && !plan->plan().coalesced) crt_groups(plan, c->h, sm, cbt, groups, group_of);
        int64_t nb = 0;
        double bf = 0, gf = 0;
        for (size_t e = 0; e < cbt.size(); e++)
            if (group_of[e] >= 0) { nb++; bf += 2.0 * (double)cbt[e].M * (double)cbt[e].N * cbt[e].kflops; }
        for (const CrtGroupHost &G : groups) {
            double r = 0, cl = 0, k = 0;
            for (int64_t v : G.rn) r += (double)v;
            for (int64_t v : G.sn) cl += (double)v;
            for (int64_t v : G.kn) k += (double)round4(v);
            gf += 2.0 * r * cl * k;
        }
        if (ngroups) *ngroups = (int64_t)groups.size();
        if (nblocks) *nblocks = nb;
        if (grouped_flops) *grouped_flops = gf;
        if (block_flops) *block_flops = bf;
    });
}

int ltg_contract2_autotune(ltg_plan *plan, ltg_bt *c, int32_t mode, int32_t nslices, double ka,
                           double kb, double kc, int32_t reps) {
    return guard([&] {
        if (!plan) throw error(kErrBadArg, "null plan");
        if (plan->external) throw error(kErrUnsupported, "a caller-built task plan has no schedule of its own");
        check_bt(c);
        need_dev(plan->ctx);
        if (plan->ctx->capturing) throw error(kErrState, "autotuning cannot run during graph capture");
        if (reps < 1) reps = 1;
        // Distinct C-block shapes, costliest bucket first.
        std::vector<GemmTask> tasks;
        std::vector<CBlockTask> cbt;
        contract2_tasks(plan->plan(), plan->a->h, plan->b->h, c->h, ka, kb, kc, tasks, cbt);
        std::map<std::pair<int64_t, int64_t>, double> work;
        std::vector<int32_t> group_of;
        const std::vector<std::pair<int64_t, int64_t>> gshapes =
            mode == LTG_MODE_PLAIN_FP64 ? plain_group_shapes(plan, c, cbt, group_of)
                                        : std::vector<std::pair<int64_t, int64_t>>();
        if (group_of.size() != cbt.size()) group_of.assign(cbt.size(), -1);
        for (size_t e = 0; e < cbt.size(); e++)
            if (group_of[e] < 0) work[{cbt[e].M, cbt[e].N}] += (double)cbt[e].M * cbt[e].N * cbt[e].kflops;
        for (const auto &g : gshapes) work[g] += (double)g.first * g.second;
        std::vector<std::pair<double, std::pair<int64_t, int64_t>>> order;
        for (auto &w : work) order.push_back({w.second, w.first});
        std::sort(order.rbegin(), order.rend());
        plan->forced_tile = -1;
        cudaStream_t s = plan->ctx->stream;
        cudaEvent_t e0, e1;
        LTG_CUDA(cudaEventCreate(&e0));
        LTG_CUDA(cudaEventCreate(&e1));
        auto timed = [&]() {
            plan->exec.clear();
            plan->sym.clear();
            int st = ltg_contract2(plan, c, mode, nslices, ka, kb, kc, 0, 0.0);   // warm + upload
            if (st != kOk) throw error(st, g_last_error);
            LTG_CUDA(cudaEventRecord(e0, s));
            for (int r = 0; r < reps; r++) {
                st = ltg_contract2(plan, c, mode, nslices, ka, kb, kc, 0, 0.0);
                if (st != kOk) throw error(st, g_last_error);
            }
            LTG_CUDA(cudaEventRecord(e1, s));
            LTG_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            LTG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            return (double)ms;
        };
        for (auto &o : order) {
            auto key = o.second;
            double best = 1e300;
            int bestc = pick_tile(key.first, key.second);
            for (int cfg = 0; cfg < tile_cfg_count(); cfg++) {
                plan->tile_override[key] = cfg;
                double ms = timed();
                if (ms < best) { best = ms; bestc = cfg; }
            }
            plan->tile_override[key] = bestc;
        }
        plan->exec.clear();
        plan->sym.clear();
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    });
}

int ltg_plan_tiles(ltg_plan *plan, int64_t *m, int64_t *n, int32_t *cfg, int64_t cap, int64_t *count) {
    return guard([&] {
        if (!plan) throw error(kErrBadArg, "null plan");
        int64_t k = 0;
        for (auto &t : plan->tile_override) {
            if (k < cap) {
                if (m) m[k] = t.first.first;
                if (n) n[k] = t.first.second;
                if (cfg) cfg[k] = t.second;
            }
            k++;
        }
        if (count) *count = k;
    });
}

int ltg_copy(ltg_bt *a, const int32_t *perm, double c, ltg_bt *b, int32_t add, double d) {
    return guard([&] {
        check_bt(a);
        need_dev(a->ctx); check_bt(b);
        run_transfer(a->ctx, {a}, {perm_from(a->h.bis.n, perm)}, {c}, b, add != 0, d);
    });
}

int ltg_add(int32_t nterms, ltg_bt *const *a, const int32_t *perms, const double *coeffs, ltg_bt *b,
            int32_t add, double d) {
    return guard([&] {
        check_bt(b);
        need_dev(b->ctx);
        if (nterms < 1 || !a || !coeffs) throw error(kErrBadArg, "add needs at least one operand");
        std::vector<ltg_bt *> srcs;
        std::vector<Perm> ps;
        std::vector<double> cs;
        for (int t = 0; t < nterms; t++) {
            check_bt(a[t]);
            srcs.push_back(a[t]);
            ps.push_back(perm_from(b->h.bis.n, perms ? perms + (size_t)t * b->h.bis.n : nullptr));
            cs.push_back(coeffs[t]);
        }
        run_transfer(b->ctx, srcs, ps, cs, b, add != 0, d);
    });
}

int ltg_dotprod_async(ltg_bt *a, const int32_t *perma, ltg_bt *b, const int32_t *permb, double *dev_out) {
    return guard([&] {
        check_bt(a);
        need_dev(a->ctx); check_bt(b);
        if (a->ctx != b->ctx) throw error(kErrBadArg, "operands belong to different contexts");
        DotExec *ex = prepare_dot(a, perm_from(a->h.bis.n, perma), b, perm_from(b->h.bis.n, permb));
        TimedLaunch tl(a->ctx, LTG_KERNEL_DOT);
        LTG_CUDA(launch_dot(ex->jobs.as<DJob>(), ex->terms.as<DTerm>(), ex->units.as<DUnit>(), ex->nrow,
                            ex->ntiled, ex->tile_bytes, a->arena.as<double>(), b->arena.as<double>(), ex->partials.as<double>(), dev_out,
                            a->ctx->stream));
        tl.done();
        a->ctx->launches += 2;
    });
}

int ltg_dotprod(ltg_bt *a, const int32_t *perma, ltg_bt *b, const int32_t *permb, double *out) {
    int st = ltg_dotprod_async(a, perma, b, permb, a ? a->ctx->dot_out.as<double>() : nullptr);
    if (st != kOk) return st;
    return guard([&] {
        if (!out) throw error(kErrBadArg, "null output");
        LTG_CUDA(cudaMemcpyAsync(out, a->ctx->dot_out.p, sizeof(double), cudaMemcpyDeviceToHost, a->ctx->stream));
        LTG_CUDA(cudaStreamSynchronize(a->ctx->stream));
    });
}

int ltg_scale(ltg_bt *a, double c) {
    return guard([&] {
        check_bt(a);
        need_dev(a->ctx);
        TimedLaunch tl(a->ctx, LTG_KERNEL_SCALE);
        LTG_CUDA(launch_scale(a->arena.as<double>(), a->h.total_elems, c, a->ctx->stream));
        tl.done();
        a->ctx->launches++;
    });
}

int ltg_denominator(ltg_bt *a, const double *eps_host, int32_t nocc) {
    return guard([&] {
        check_bt(a);
        need_dev(a->ctx);
        if (a->h.bis.n != 4) throw error(kErrUnsupported, "denominator is defined for 4-index tensors");
        if (!eps_host) throw error(kErrBadArg, "null orbital energies");
        int64_t tot = 0;
        std::vector<int64_t> off(kDevMaxOrder, 0);
        for (int d = 0; d < 4; d++) { off[d] = tot; tot += a->h.bis.dims[d]; }
        std::vector<double> eps(eps_host, eps_host + tot);
        if (eps != a->denom_eps || nocc != a->denom_nocc || !a->dir_uploaded) {
            if (a->ctx->capturing)
                throw error(kErrState, "denominator not prepared before graph capture: call it once outside the capture");
            upload_directory(a);
            upload_vec(a->denom_dev, eps, a->ctx->stream);
            upload_vec(a->denom_off, off, a->ctx->stream);
            a->denom_eps = eps;
            a->denom_nocc = nocc;
        }
        TimedLaunch tl(a->ctx, LTG_KERNEL_DENOMINATOR);
        LTG_CUDA(launch_denominator(a->arena.as<double>(), a->dir_off.as<int64_t>(), a->dir_start.as<int64_t>(),
                                    a->dir_ext.as<int32_t>(), (int32_t)a->h.blk_abs.size(), a->denom_dev.as<double>(),
                                    a->denom_off.as<int64_t>(), nocc, a->ctx->stream));
        tl.done();
        a->ctx->launches++;
    });
}

int ltg_graph_begin(ltg_ctx *ctx) {
    return guard([&] {
        check_ctx(ctx);
        need_dev(ctx);
        if (ctx->capturing) throw error(kErrState, "capture already active");
        LTG_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        ctx->capturing = true;
    });
}

int ltg_graph_end(ltg_ctx *ctx, ltg_graph **out) {
    return guard([&] {
        check_ctx(ctx);
        if (!ctx->capturing) throw error(kErrState, "no capture active");
        ctx->capturing = false;
        std::unique_ptr<ltg_graph> g(new ltg_graph());
        g->ctx = ctx;
        LTG_CUDA(cudaStreamEndCapture(ctx->stream, &g->graph));
        LTG_CUDA(cudaGraphInstantiate(&g->exec, g->graph, 0));
        if (out) *out = g.release();
    });
}

int ltg_graph_launch(ltg_graph *g) {
    return guard([&] {
        if (!g) throw error(kErrBadArg, "null graph");
        LTG_CUDA(cudaGraphLaunch(g->exec, g->ctx->stream));
    });
}

int ltg_graph_destroy(ltg_graph *g) {
    return guard([&] {
        if (!g) throw error(kErrBadArg, "null graph");
        if (g->exec) cudaGraphExecDestroy(g->exec);
        if (g->graph) cudaGraphDestroy(g->graph);
        delete g;
    });
}

}  // extern "C"
