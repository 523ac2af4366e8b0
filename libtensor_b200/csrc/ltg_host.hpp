// Host-side engine of the B200 block-tensor path: block index spaces,
// symmetry (permutational anti/symmetry, partitions, point-group labels),
// orbits, the btod_contract2 schedule (non-zero C orbits and per-block
// contraction pair lists) and the flat task lists uploaded to the GPU.
//
// All integer work here is bit-exact with respect to the reference
// (libtensor): orbits are enumerated with the same breadth-first rule and the
// canonical block is the minimum absolute index in its orbit
// (libtensor/core/impl/orbit_impl.h:139-297,
//  libtensor/core/impl/short_orbit_impl.h:91-153).
#pragma once

#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace ltg {

constexpr int kMaxOrder = 8;
constexpr int kMaxTerms_host = 8;   // operands of one btod_add pass

struct error : std::runtime_error {
    int code;
    error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// Status codes shared with the C ABI (include/ltg.h).
enum {
    kOk = 0,
    kErrBadArg = 1,
    kErrBadDims = 2,
    kErrSymmetry = 3,
    kErrUnsupported = 4,
    kErrOom = 5,
    kErrCuda = 6,
    kErrTimeout = 7,
    kErrState = 8,
};

// Permutation in the reference's convention
// (libtensor/core/permutation.h): applying it to a sequence s gives
// s'[i] = s[p[i]]; permute(q) composes "this, then q": r[i] = p[q[i]].
struct Perm {
    int n = 0;
    int8_t p[kMaxOrder] = {0, 1, 2, 3, 4, 5, 6, 7};

    static Perm identity(int n) { Perm r; r.n = n; return r; }
    bool is_identity() const {
        for (int i = 0; i < n; i++) if (p[i] != i) return false;
        return true;
    }
    template<class T> void apply(T *s) const {
        T buf[kMaxOrder];
        for (int i = 0; i < n; i++) buf[i] = s[i];
        for (int i = 0; i < n; i++) s[i] = buf[p[i]];
    }
    Perm &permute(const Perm &q) {
        int8_t cp[kMaxOrder];
        for (int i = 0; i < n; i++) cp[i] = p[i];
        for (int i = 0; i < n; i++) p[i] = cp[q.p[i]];
        return *this;
    }
    Perm inverse() const {
        Perm r; r.n = n;
        for (int i = 0; i < n; i++) r.p[p[i]] = (int8_t)i;
        return r;
    }
    bool operator==(const Perm &o) const {
        if (n != o.n) return false;
        for (int i = 0; i < n; i++) if (p[i] != o.p[i]) return false;
        return true;
    }
    bool operator!=(const Perm &o) const { return !(*this == o); }
};

// Block transformation: permutation of indices plus a scalar factor
// (libtensor/core/tensor_transf.h).
struct Transf {
    Perm perm;
    double coeff = 1.0;
    static Transf identity(int n) { Transf t; t.perm = Perm::identity(n); return t; }
    Transf &transform(const Transf &t) { perm.permute(t.perm); coeff *= t.coeff; return *this; }
    Transf &invert() { perm = perm.inverse(); coeff = 1.0 / coeff; return *this; }
};

// Block index space: each dimension split into blocks at given positions
// (libtensor/core/block_index_space.h).
struct Bis {
    int n = 0;
    int64_t dims[kMaxOrder] = {};
    int type[kMaxOrder] = {};
    std::vector<int64_t> starts[kMaxOrder];   // block start positions, starts[d][0] == 0
    int64_t bidims[kMaxOrder] = {};           // number of blocks per dimension

    void finalize();
    int64_t nblocks() const {
        int64_t r = 1;
        for (int d = 0; d < n; d++) r *= bidims[d];
        return r;
    }
    int64_t block_extent(int d, int64_t b) const {
        const std::vector<int64_t> &s = starts[d];
        return (b + 1 < (int64_t)s.size() ? s[b + 1] : dims[d]) - s[b];
    }
    void block_dims(const int64_t *bidx, int64_t *out) const {
        for (int d = 0; d < n; d++) out[d] = block_extent(d, bidx[d]);
    }
    int64_t block_size(const int64_t *bidx) const {
        int64_t r = 1;
        for (int d = 0; d < n; d++) r *= block_extent(d, bidx[d]);
        return r;
    }
    int64_t abs(const int64_t *bidx) const {
        int64_t a = 0;
        for (int d = 0; d < n; d++) a = a * bidims[d] + bidx[d];
        return a;
    }
    void unabs(int64_t a, int64_t *bidx) const {
        for (int d = n - 1; d >= 0; d--) { bidx[d] = a % bidims[d]; a /= bidims[d]; }
    }
    Bis permuted(const Perm &p) const;
    bool equals(const Bis &o) const;
};

// se_perm: one generator of the permutational (anti)symmetry group
// (libtensor/symmetry/se_perm.h:28-140).
struct SePerm {
    Perm perm;
    double coeff;
};

// se_part without partition maps: forbidden partitions only
// (libtensor/symmetry/se_part.h:32; mark_forbidden and is_allowed at
// libtensor/symmetry/inst/se_part_impl.h:189-296).  Partition maps
// (add_map) are rejected with kErrUnsupported.
struct SePart {
    int64_t pdims[kMaxOrder] = {};    // partitions per dimension (1 = unaffected)
    int64_t bipdims[kMaxOrder] = {};  // blocks per partition per dimension
    std::vector<char> forbidden;      // by absolute partition index
    bool is_allowed(int n, const int64_t *bidx) const {
        int64_t a = 0;
        for (int d = 0; d < n; d++) a = a * pdims[d] + bidx[d] / bipdims[d];
        return !forbidden[a];
    }
};

// One term of a label product rule: multiset of dimensions (multiplicity per
// dimension) whose block labels are multiplied, and the intrinsic label the
// product must contain (libtensor/symmetry/product_rule.h).
struct LabelTerm {
    uint8_t seq[kMaxOrder] = {};
    int intr = 0;
};

// se_label for abelian groups whose irreps multiply as XOR (C1, Ci, Cs, C2,
// C2h, C2v, D2, D2h with the usual numbering).  The rule is an OR over
// products, each an AND over terms (libtensor/symmetry/inst/se_label_impl.h:74-112).
struct SeLabel {
    int nirrep = 1;
    std::vector<int> labels[kMaxOrder];          // per dim per block, -1 = unlabelled
    std::vector<std::vector<LabelTerm>> rule;    // OR of AND-products
    bool is_allowed(int n, const int64_t *bidx) const;
};

struct Symmetry {
    std::vector<SePerm> perm;
    std::vector<SePart> part;
    std::vector<SeLabel> label;
    bool is_allowed(int n, const int64_t *bidx) const {
        for (const SePart &p : part) if (!p.is_allowed(n, bidx)) return false;
        for (const SeLabel &l : label) if (!l.is_allowed(n, bidx)) return false;
        return true;
    }
};

// Orbit of one block: members sorted by absolute index with the transform
// taking the canonical block to each member.
struct Orbit {
    int64_t canonical = 0;
    bool allowed = true;
    std::vector<std::pair<int64_t, Transf>> members;   // sorted by index
    const Transf *find(int64_t aidx) const;
};

// Builds the orbit of block aidx with the reference's breadth-first rule.
void build_orbit(const Bis &bis, const Symmetry &sym, int64_t aidx, Orbit &o);

// Per-block orbit table of a whole block index space: canonical index,
// transform canonical -> block, allowed flag.  Built once per symmetry.
struct OrbitTable {
    std::vector<int64_t> canon;    // canonical abs index for each block
    std::vector<Transf> tr;        // transform canonical -> block
    std::vector<char> allowed;     // orbit allowed
    std::vector<int64_t> canon_list;  // all canonical allowed blocks, ascending
    void build(const Bis &bis, const Symmetry &sym);
};

// Contraction descriptor with the reference's index-connection bookkeeping
// (libtensor/core/contraction2.h:48-330): conn has 2*(N+M+K) slots laid out
// as [C indices | A indices | B indices]; each slot holds the slot it is
// connected to.
struct Contraction {
    int N = 0, M = 0, K = 0;
    Perm permc;
    int64_t conn[3 * kMaxOrder] = {};
    int nk_set = 0;

    void init(int n, int m, int k, const Perm &pc);
    void contract(int ia, int ib);
    void permute_a(const Perm &pa);
    void permute_b(const Perm &pb);
    void permute_c(const Perm &pc);
    bool same_conn(const Contraction &o) const {
        int tot = 2 * (N + M + K);
        for (int i = 0; i < tot; i++) if (conn[i] != o.conn[i]) return false;
        return true;
    }
    int NA() const { return N + K; }
    int NB() const { return M + K; }
    int NC() const { return N + M; }
private:
    void connect();
    void make_seqc(int64_t *seqc) const;
    void adjust_permc(const int64_t *seqc1, const int64_t *seqc2);
};

// One entry of a contraction pair list (gen_bto_contract2_pair,
// libtensor/gen_block_tensor/gen_bto_contract2_clst.h:23-128).
struct Pair {
    int64_t aia, acia, aib, acib;
    Transf tra, trb;
};

// Block tensor host state: bis, symmetry, orbit table, canonical block
// directory (offset of each stored canonical block in the device arena) and
// the non-zero flags.
struct BlockTensorHost {
    Bis bis;
    Symmetry sym;
    OrbitTable orbits;
    std::vector<int64_t> blk_abs;     // canonical allowed blocks, ascending
    std::vector<int64_t> blk_off;     // element offset of each in the arena
    std::vector<int64_t> blk_size;    // elements per block
    std::vector<char> nonzero;        // per stored block
    std::vector<int64_t> slot_of;     // abs index -> stored slot or -1
    int64_t total_elems = 0;
    void build_directory();
    int64_t slot(int64_t aidx) const { return slot_of[aidx]; }
};

// ------------------------------------------------------------------------
// btod_contract2 plan: schedule of non-zero canonical C blocks and, for
// each, the coalesced pair list converted to GEMM tasks over the arenas.

// Strided sub-dimension groups of one matricised operand after loop fusion.
constexpr int kMaxSub = 4;
struct SubDims {
    int n = 0;
    int32_t ext[kMaxSub] = {};
    int64_t s0[kMaxSub] = {};   // stride in the first tensor of the pair
    int64_t s1[kMaxSub] = {};   // stride in the second tensor of the pair
    int64_t total() const { int64_t r = 1; for (int i = 0; i < n; i++) r *= ext[i]; return r; }
};

// One GEMM-shaped product of a (C block, coalesced pair):
//   C[m,n] (+)= coeff * sum_k A[m,k] * B[n,k]
// with m over (C dims taken from A), n over (C dims taken from B), k over the
// contracted pairs; offsets are in elements of each tensor's arena.
struct GemmTask {
    int64_t c_off, a_off, b_off;
    SubDims m;   // s0: stride in A, s1: stride in C
    SubDims n;   // s0: stride in B, s1: stride in C
    SubDims k;   // s0: stride in A, s1: stride in B
    double coeff;
    int32_t cblk;   // index into the C-block list of the plan
};

// Per scheduled C block: output mapping (C strides only) and task range.
struct CBlockTask {
    int64_t c_off = 0;
    int64_t M = 1, N = 1;
    SubDims cm, cn;               // s0 = s1 = stride in C
    int32_t t_begin = 0, t_end = 0;
    double coeff0 = 1.0;          // coefficient of the first task
    double kflops = 0;            // sum over tasks of K (work estimate)
};

struct ContractPlan {
    Contraction contr;
    Bis bisc;
    Symmetry symc;
    std::vector<int64_t> schedule;                 // non-zero canonical C blocks
    std::vector<std::vector<Pair>> clst;           // coalesced pairs per schedule entry
    double flops = 0;                              // algorithmic flops (2*|C|*K per pair)
    bool coalesced = false;                        // some pair list was shortened by coalescing
};

// Derives the result block index space and symmetry
// (gen_bto_contract2_bis / gen_bto_contract2_sym:
//  libtensor/gen_block_tensor/impl/gen_bto_contract2_sym_impl.h:42-83).
void contract2_result_space(const Contraction &c, const BlockTensorHost &a,
    const BlockTensorHost &b, Bis &bisc, Symmetry &symc);

// Builds the schedule and coalesced pair lists
// (gen_bto_contract2_nzorb::build, gen_bto_contract2_nzorb_impl.h:354-477;
//  gen_bto_contract2_clst_builder::build_list, *_clst_builder_impl.h:188-323;
//  btod_contract2_clst_optimize::perform, btod_contract2_clst_optimize_impl.h:11-56).
void contract2_schedule(const Contraction &c, const BlockTensorHost &a,
    const BlockTensorHost &b, ContractPlan &plan, int nthreads);

// Converts the plan into GEMM tasks against concrete arenas of A, B and C
// (gen_bto_contract2_block::compute_block, *_block_impl.h:100-205, then the
// index mapping of tod_contract2).
void contract2_tasks(const ContractPlan &plan, const BlockTensorHost &a,
    const BlockTensorHost &b, const BlockTensorHost &c, double ka, double kb,
    double kc, std::vector<GemmTask> &tasks, std::vector<CBlockTask> &cblocks);

// Permuted block index space and symmetry: the space of P(A) for
// B[y] = A[x] with y[d] = x[perm[d]] (so_permute).
void permute_space(const Bis &bis, const Symmetry &sym, const Perm &p, Bis &out_bis,
                   Symmetry &out_sym);

// Transfer/dot planning for btod_copy / btod_add / btod_dotprod.
struct TransferTerm {
    const BlockTensorHost *src;
    Perm perm;
    double coeff;
    int32_t src_index;
};
struct TJob {
    int64_t dst_off;
    int32_t ndim, inner;
    int32_t nterms, term0;
    int32_t ext[kMaxOrder];
};
struct TTerm {
    int64_t src_off;
    double coeff;
    int32_t src, pad;
    int32_t sstr[kMaxOrder];
};
struct TUnit {
    int32_t job, pad;
    int64_t row_begin, row_end;
};
struct TransferPlan {
    std::vector<TJob> jobs;
    std::vector<TTerm> terms;
    std::vector<TUnit> units;
    std::vector<char> dst_nonzero;     // per destination slot: any term contributed
    double bytes = 0;                  // algorithmic bytes moved
};
void plan_transfer(const std::vector<TransferTerm> &terms, const BlockTensorHost &dst,
                   bool accumulate, TransferPlan &plan);
void plan_dot(const BlockTensorHost &a, const Perm &pa, const BlockTensorHost &b,
              const Perm &pb, TransferPlan &plan);
std::vector<SePerm> perm_group_closure(int n, const std::vector<SePerm> &gens);

// Element-wise transfer task: dst block (+)= coeff * P(src block)
// (tod_copy / tod_add through gen_bto_copy / gen_bto_add).
struct CopyTask {
    int64_t dst_off, src_off;
    int32_t ndim;
    int32_t ext[kMaxOrder];       // destination block extents
    int64_t sstr[kMaxOrder];      // source stride for each destination dim
    double coeff;
    int32_t src_tensor;           // operand index (multi-term add)
};

}  // namespace ltg
