/*
 * ref_driver.C -- C entry points around the reference implementation
 * (libtensor) of the block-sparse contraction path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is compiled together with the
 * reference's own sources (see Makefile) into oracle/_ref/libltref.so.  The
 * parity tests and the CPU-baseline leg of bench.py load it through ctypes;
 * product code never does.
 *
 * What it exposes, all through the reference's public classes:
 *   - block tensors with se_perm / se_part / se_label symmetry
 *     (libtensor/block_tensor/block_tensor.h:22, symmetry/se_perm.h:28,
 *      symmetry/se_part.h:32, symmetry/se_label.h:37);
 *   - btod_contract2<N,M,K> construction, schedule and perform
 *     (libtensor/block_tensor/btod_contract2.h:29-140);
 *   - the per-C-block contraction pair list exactly as the schedule builder
 *     makes it (gen_block_tensor/impl/gen_bto_contract2_nzorb_impl.h:455-463
 *     calls gen_bto_contract2_clst_builder::build_list(false, cbl));
 *   - the schedule's work as the reference's task cost counts it
 *     (gen_block_tensor/impl/gen_bto_contract2_block_impl.h:63-95);
 *   - btod_copy / btod_add / btod_dotprod (block_tensor/btod_copy.h:38,
 *     btod_add.h:38, btod_dotprod.h:35);
 *   - seeded test inputs written straight into the reference's tensors (the
 *     same distribution as the product's input generator, restated here), so
 *     that a CPU-only caller needs nothing but this library.
 *
 * Tensor description ("spec") is a flat int64 array; the layout is documented
 * at parse_spec() and produced by oracle/refapi.py.
 */
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#include <stdexcept>
#include <sys/time.h>
#include <thread>

#include <libutil/thread_pool/thread_pool.h>
#include <libtensor/core/allocator.h>
#include <libtensor/core/abs_index.h>
#include <libtensor/core/orbit.h>
#include <libtensor/core/orbit_list.h>
#include <libtensor/core/short_orbit.h>
#include <libtensor/core/batching_policy_base.h>
#include <libtensor/block_tensor/block_tensor.h>
#include <libtensor/block_tensor/block_tensor_ctrl.h>
#include <libtensor/block_tensor/btod_contract2.h>
#include <libtensor/block_tensor/btod_add.h>
#include <libtensor/block_tensor/btod_copy.h>
#include <libtensor/block_tensor/btod_dotprod.h>
#include <libtensor/block_tensor/btod_symmetrize2.h>
#include <libtensor/block_tensor/btod_symmetrize4.h>
#include <libtensor/dense_tensor/dense_tensor_ctrl.h>
#include <libtensor/symmetry/so_copy.h>
#include <libtensor/symmetry/se_perm.h>
#include <libtensor/symmetry/se_part.h>
#include <libtensor/symmetry/se_label.h>
#include <libtensor/symmetry/point_group_table.h>
#include <libtensor/symmetry/product_table_container.h>
#include <libtensor/gen_block_tensor/impl/gen_bto_contract2_clst_builder.h>
#include <libtensor/gen_block_tensor/impl/gen_bto_contract2_block_list.h>
#include <libtensor/gen_block_tensor/impl/gen_bto_unfold_block_list.h>
#include <libtensor/block_tensor/btod_traits.h>
#include <libtensor/gen_block_tensor/gen_block_tensor_ctrl.h>

extern "C" void openblas_set_num_threads(int);

using namespace libtensor;

namespace {

using libtensor::index;

std::string g_err;
std::unique_ptr<libutil::thread_pool> g_pool;

typedef allocator<double> alloc_t;

/* ---- point-group tables: abelian groups whose irreps multiply as XOR ---- */
std::string ensure_xor_table(int nirrep) {
    std::string id = "ltg_xor" + std::to_string(nirrep);
    product_table_container &ptc = product_table_container::get_instance();
    if (ptc.table_exists(id)) return id;
    std::vector<std::string> names(nirrep);
    for (int i = 0; i < nirrep; i++) names[i] = "G" + std::to_string(i);
    point_group_table pg(id, names, names[0]);
    for (int a = 0; a < nirrep; a++)
        for (int b = a; b < nirrep; b++)
            if (a != 0 && b != 0) pg.add_product(a, b, a ^ b);
    pg.check();
    ptc.add(pg);
    return id;
}

struct bt_base {
    size_t order;
    virtual ~bt_base() {}
};

template<size_t N>
struct bt_h : bt_base {
    block_index_space<N> bis;
    block_tensor<N, double, alloc_t> bt;
    explicit bt_h(const block_index_space<N> &b) : bis(b), bt(b) { this->order = N; }
};

/*
 * Spec layout (all int64):
 *   N
 *   dims[N]
 *   dim_type[N]                       (dims with equal type share splits)
 *   for each type t = 0..max(dim_type): nsplit, split positions...
 *   nperm;   per generator: perm[N] (libtensor convention), sign (+1/-1)
 *   npart;   per se_part: pdims[N],
 *                         nforbidden, forbidden partition indices [nforb*N],
 *                         nmaps, maps [(from[N], to[N], sign) * nmaps]
 *   nlabel;  per se_label: nirrep (XOR table), per dim: nblk_d, labels[nblk_d]
 *                          (label -1 = unlabelled), nintr, intrinsic labels
 * Symmetry elements are inserted in that order: perm, part, label.
 */
struct spec_reader {
    const int64_t *p; size_t n, i;
    int64_t next() {
        if (i >= n) throw std::runtime_error("spec truncated");
        return p[i++];
    }
};

template<size_t N>
permutation<N> perm_from(const int32_t *p) {
    // p[d] = index of the source position that lands at position d, i.e. the
    // libtensor permutation whose operator[](d) == p[d].
    permutation<N> perm;
    if (!p) return perm;
    // Compose transpositions to reach the target m_idx (selection sort).
    size_t cur[N];
    for (size_t d = 0; d < N; d++) cur[d] = d;
    for (size_t d = 0; d < N; d++) {
        if (cur[d] == (size_t)p[d]) continue;
        size_t j = d + 1;
        while (j < N && cur[j] != (size_t)p[d]) j++;
        perm.permute(d, j);
        std::swap(cur[d], cur[j]);
    }
    return perm;
}

template<size_t N>
bt_h<N> *make_bt(spec_reader &r) {
    index<N> i1, i2;
    int64_t dims[N], types[N];
    for (size_t d = 0; d < N; d++) { dims[d] = r.next(); i2[d] = dims[d] - 1; }
    int64_t ntypes = 0;
    for (size_t d = 0; d < N; d++) {
        types[d] = r.next();
        if (types[d] + 1 > ntypes) ntypes = types[d] + 1;
    }
    dimensions<N> dd(index_range<N>(i1, i2));
    block_index_space<N> bis(dd);
    for (int64_t t = 0; t < ntypes; t++) {
        mask<N> m;
        for (size_t d = 0; d < N; d++) m[d] = (types[d] == t);
        int64_t ns = r.next();
        for (int64_t s = 0; s < ns; s++) bis.split(m, (size_t)r.next());
    }
    bt_h<N> *h = new bt_h<N>(bis);
    dimensions<N> bidims = bis.get_block_index_dims();
    block_tensor_wr_ctrl<N, double> ctrl(h->bt);
    symmetry<N, double> &sym = ctrl.req_symmetry();

    int64_t nperm = r.next();
    for (int64_t g = 0; g < nperm; g++) {
        int32_t pv[N];
        for (size_t d = 0; d < N; d++) pv[d] = (int32_t)r.next();
        double sign = (double)r.next();
        sym.insert(se_perm<N, double>(perm_from<N>(pv),
            scalar_transf<double>(sign)));
    }

    int64_t npart = r.next();
    for (int64_t e = 0; e < npart; e++) {
        index<N> p1, p2;
        for (size_t d = 0; d < N; d++) p2[d] = (size_t)r.next() - 1;
        dimensions<N> pdims(index_range<N>(p1, p2));
        se_part<N, double> sp(bis, pdims);
        int64_t nmaps_or_forb = r.next();
        std::vector< index<N> > forb;
        for (int64_t f = 0; f < nmaps_or_forb; f++) {
            index<N> fi;
            for (size_t d = 0; d < N; d++) fi[d] = (size_t)r.next();
            forb.push_back(fi);
        }
        int64_t nmaps = r.next();
        for (int64_t m = 0; m < nmaps; m++) {
            index<N> a, b;
            for (size_t d = 0; d < N; d++) a[d] = (size_t)r.next();
            for (size_t d = 0; d < N; d++) b[d] = (size_t)r.next();
            double sign = (double)r.next();
            sp.add_map(a, b, scalar_transf<double>(sign));
        }
        for (size_t f = 0; f < forb.size(); f++) sp.mark_forbidden(forb[f]);
        sym.insert(sp);
    }

    int64_t nlabel = r.next();
    for (int64_t e = 0; e < nlabel; e++) {
        int nirrep = (int)r.next();
        std::string id = ensure_xor_table(nirrep);
        se_label<N, double> sl(bidims, id);
        block_labeling<N> &bl = sl.get_labeling();
        std::vector< std::vector<int64_t> > labs(N);
        for (size_t d = 0; d < N; d++) {
            int64_t nb = r.next();
            for (int64_t b = 0; b < nb; b++) labs[d].push_back(r.next());
        }
        // dims with the same labels are labelled together (one mask), so that
        // they keep one dimension type in the labeling (symmetrizers over
        // them require it, so_symmetrize_se_label_impl.h:53-62)
        std::vector<bool> done(N, false);
        for (size_t d = 0; d < N; d++) {
            if (done[d]) continue;
            mask<N> m;
            for (size_t e2 = d; e2 < N; e2++)
                if (!done[e2] && labs[e2] == labs[d] && bidims[e2] == bidims[d]) { m[e2] = true; done[e2] = true; }
            for (size_t b = 0; b < labs[d].size(); b++)
                if (labs[d][b] >= 0) bl.assign(m, b, (size_t)labs[d][b]);
        }
        int64_t nintr = r.next();
        product_table_i::label_set_t ls;
        for (int64_t k = 0; k < nintr; k++) ls.insert((size_t)r.next());
        sl.set_rule(ls);
        sym.insert(sl);
    }
    return h;
}

template<size_t N>
bt_h<N> *as(void *h) {
    bt_base *b = static_cast<bt_base*>(h);
    if (b->order != N) throw std::runtime_error("tensor order mismatch");
    return static_cast<bt_h<N>*>(b);
}

template<size_t N>
index<N> to_index(const int64_t *bidx) {
    index<N> i;
    for (size_t d = 0; d < N; d++) i[d] = (size_t)bidx[d];
    return i;
}

template<size_t N>
void perm_to(const permutation<N> &p, int32_t *out) {
    for (size_t d = 0; d < N; d++) out[d] = (int32_t)p[d];
}

/* ---------------- block tensor entry points, dispatched on order ------- */

template<size_t N>
int set_block(void *h, const int64_t *bidx, const double *data, size_t n) {
    bt_h<N> *t = as<N>(h);
    index<N> idx = to_index<N>(bidx);
    dimensions<N> bd = t->bis.get_block_dims(idx);
    if (bd.get_size() != n) throw std::runtime_error("block size mismatch");
    block_tensor_wr_ctrl<N, double> ctrl(t->bt);
    dense_tensor_wr_i<N, double> &blk = ctrl.req_block(idx);
    {
        dense_tensor_wr_ctrl<N, double> tc(blk);
        double *p = tc.req_dataptr();
        std::memcpy(p, data, n * sizeof(double));
        tc.ret_dataptr(p);
    }
    ctrl.ret_block(idx);
    return 0;
}

template<size_t N>
int get_block(void *h, const int64_t *bidx, double *data, size_t n) {
    bt_h<N> *t = as<N>(h);
    index<N> idx = to_index<N>(bidx);
    dimensions<N> bd = t->bis.get_block_dims(idx);
    if (bd.get_size() != n) throw std::runtime_error("block size mismatch");
    block_tensor_rd_ctrl<N, double> ctrl(t->bt);
    if (ctrl.req_is_zero_block(idx)) {
        std::memset(data, 0, n * sizeof(double));
        return 1;
    }
    dense_tensor_rd_i<N, double> &blk = ctrl.req_const_block(idx);
    {
        dense_tensor_rd_ctrl<N, double> tc(blk);
        const double *p = tc.req_const_dataptr();
        std::memcpy(data, p, n * sizeof(double));
        tc.ret_const_dataptr(p);
    }
    ctrl.ret_const_block(idx);
    return 0;
}

template<size_t N>
size_t nonzero(void *h, int64_t *out, size_t cap) {
    bt_h<N> *t = as<N>(h);
    gen_block_tensor_rd_ctrl<N, block_tensor_i_traits<double> > ctrl(t->bt);
    std::vector<size_t> v;
    ctrl.req_nonzero_blocks(v);
    for (size_t i = 0; i < v.size() && i < cap; i++) out[i] = (int64_t)v[i];
    return v.size();
}

template<size_t N>
void block_index_dims(void *h, int64_t *out) {
    bt_h<N> *t = as<N>(h);
    dimensions<N> bd = t->bis.get_block_index_dims();
    for (size_t d = 0; d < N; d++) out[d] = (int64_t)bd[d];
}

template<size_t N>
int orbit_info(void *h, int64_t aidx, int64_t *canon, int32_t *perm,
    double *coeff, int64_t *orbit_size) {
    bt_h<N> *t = as<N>(h);
    block_tensor_rd_ctrl<N, double> ctrl(t->bt);
    const symmetry<N, double> &sym = ctrl.req_const_symmetry();
    orbit<N, double> o(sym, (size_t)aidx, true);
    *canon = (int64_t)o.get_acindex();
    const tensor_transf<N, double> &tr = o.get_transf((size_t)aidx);
    perm_to<N>(tr.get_perm(), perm);
    *coeff = tr.get_scalar_tr().get_coeff();
    size_t cnt = 0;
    for (typename orbit<N, double>::iterator i = o.begin(); i != o.end(); ++i) cnt++;
    *orbit_size = (int64_t)cnt;
    return o.is_allowed() ? 1 : 0;
}

/* ---------------- seeded test inputs ------------------------------------ */

/* The test-input distribution, restated: splitmix64 (Steele, Lea & Flood,
   OOPSLA 2014) keyed by the element's linear index in the full dense tensor,
   six 64-bit draws giving twelve 32-bit uniforms, centred sum; symmetrised as
   sum over the group (perm, sign) of sign * g(P x); one final multiply by
   scale * 2^-32. */
inline uint64_t sm64_mix(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

inline int64_t seeded_int(uint64_t seed, uint64_t lin) {
    uint64_t key = sm64_mix(seed), s = 0;
    for (int r = 0; r < 6; r++) {
        uint64_t h = sm64_mix(key + lin * 6u + (uint64_t)r);
        s += (h & 0xffffffffULL) + (h >> 32);
    }
    return (int64_t)s - (int64_t)(6ULL << 32);
}

/* Fills every canonical, allowed block of the tensor (the reference's own
   orbit_list) with the seeded values; elements of a block are spread over
   nthreads host threads. */
template<size_t N>
void fill_seeded(void *h, uint64_t seed, double scale, int ng,
    const int32_t *perms, const int32_t *signs, int nthreads) {
    bt_h<N> *t = as<N>(h);
    block_tensor_wr_ctrl<N, double> ctrl(t->bt);
    orbit_list<N, double> ol(ctrl.req_const_symmetry());
    const dimensions<N> &dims = t->bis.get_dims();
    const double sc = scale * 0x1p-32;
    if (nthreads < 1) nthreads = 1;
    for (typename orbit_list<N, double>::iterator it = ol.begin();
         it != ol.end(); ++it) {
        index<N> bi;
        ol.get_index(it, bi);
        index<N> start = t->bis.get_block_start(bi);
        dimensions<N> bd = t->bis.get_block_dims(bi);
        size_t n = bd.get_size();
        dense_tensor_wr_i<N, double> &blk = ctrl.req_block(bi);
        {
            dense_tensor_wr_ctrl<N, double> tc(blk);
            double *p = tc.req_dataptr();
            auto work = [&](size_t e0, size_t e1) {
                size_t x[N];
                for (size_t e = e0; e < e1; e++) {
                    size_t r = e;
                    for (size_t d = N; d-- > 0;) {
                        x[d] = start[d] + r % bd[d];
                        r /= bd[d];
                    }
                    int64_t v = 0;
                    for (int g = 0; g < ng; g++) {
                        uint64_t lin = 0;
                        for (size_t d = 0; d < N; d++)
                            lin = lin * (uint64_t)dims[d] + (uint64_t)x[perms[g * N + d]];
                        int64_t s = seeded_int(seed, lin);
                        v += signs[g] > 0 ? s : -s;
                    }
                    p[e] = (double)v * sc;
                }
            };
            size_t nt = std::min<size_t>((size_t)nthreads, (n + 4095) / 4096);
            if (nt <= 1) {
                work(0, n);
            } else {
                std::vector<std::thread> th;
                for (size_t w = 0; w < nt; w++)
                    th.emplace_back(work, n * w / nt, n * (w + 1) / nt);
                for (auto &x : th) x.join();
            }
            tc.ret_dataptr(p);
        }
        ctrl.ret_block(bi);
    }
}

/* Orbital-energy denominator, in place: every element of every canonical
   block divided by sum_d (d < nocc ? +1 : -1) eps[eps_off[d] + x_d], the sum
   taken from the last dimension to the first (as the product's kernel does,
   so both divide by the same double).  This is caller code over the
   reference's block access, as a coupled-cluster program writes it. */
template<size_t N>
void denominator(void *h, const double *eps, int nocc) {
    bt_h<N> *t = as<N>(h);
    std::vector<size_t> nz;
    {
        gen_block_tensor_rd_ctrl<N, block_tensor_i_traits<double> > rc(t->bt);
        rc.req_nonzero_blocks(nz);
    }
    block_tensor_wr_ctrl<N, double> ctrl(t->bt);
    const dimensions<N> &dims = t->bis.get_dims();
    const dimensions<N> bidims = t->bis.get_block_index_dims();
    size_t eoff[N];
    for (size_t d = 0, o = 0; d < N; d++) { eoff[d] = o; o += dims[d]; }
    for (size_t k = 0; k < nz.size(); k++) {
        index<N> bi;
        abs_index<N>::get_index(nz[k], bidims, bi);
        index<N> start = t->bis.get_block_start(bi);
        dimensions<N> bd = t->bis.get_block_dims(bi);
        dense_tensor_wr_i<N, double> &blk = ctrl.req_block(bi);
        {
            dense_tensor_wr_ctrl<N, double> tc(blk);
            double *p = tc.req_dataptr();
            const size_t n = bd.get_size();
            for (size_t e = 0; e < n; e++) {
                size_t r = e;
                double den = 0.0;
                for (size_t d = N; d-- > 0;) {
                    const size_t x = start[d] + r % bd[d];
                    r /= bd[d];
                    const double v = eps[eoff[d] + x];
                    den += (int)d < nocc ? v : -v;
                }
                p[e] /= den;
            }
            tc.ret_dataptr(p);
        }
        ctrl.ret_block(bi);
    }
}

/* ---------------- symmetrizers ----------------------------------------- */

/* b = op + s P(op) for a unitary permutation P (btod_symmetrize2,
   block_tensor/btod_symmetrize2.h:54), or the sum over the 24 permutations
   of four indexes with the parity sign (btod_symmetrize4,
   block_tensor/btod_symmetrize4.h:53), of any additive operation op. */
// The reference instantiates btod_symmetrize2 for orders >= 2 and
// btod_symmetrize4 for orders >= 4 (block_tensor/impl/btod_symmetrize2.C,
// btod_symmetrize4.C).
template<size_t N, bool Two = (N >= 2), bool Four = (N >= 4)>
struct symm_impl {
    static void run(additive_gen_bto<N, btod_traits::bti_traits> &, int, const int32_t *, int, void *, int,
                    double) {
        throw std::runtime_error("symmetrize: tensor order too small");
    }
};
template<size_t N, bool Four>
struct symm_impl<N, true, Four> {
    static void run(additive_gen_bto<N, btod_traits::bti_traits> &op, int nidx, const int32_t *idx, int symm,
                    void *b, int add, double d) {
        block_tensor<N, double, alloc_t> &bt = as<N>(b)->bt;
        if (nidx == 2 || nidx == -1) {
            permutation<N> p;
            if (nidx == 2) p.permute((size_t)idx[0], (size_t)idx[1]);
            else p = perm_from<N>(idx);
            btod_symmetrize2<N> s(op, p, symm != 0);
            if (add) s.perform(bt, d);
            else s.perform(bt);
        } else {
            symm_impl<N, false, Four>::run(op, nidx, idx, symm, b, add, d);
        }
    }
};
template<size_t N>
struct symm_impl<N, false, true> {
    static void run(additive_gen_bto<N, btod_traits::bti_traits> &op, int nidx, const int32_t *idx, int symm,
                    void *b, int add, double d) {
        if (nidx != 4) throw std::runtime_error("symmetrize: 2 or 4 indexes, or a permutation");
        block_tensor<N, double, alloc_t> &bt = as<N>(b)->bt;
        btod_symmetrize4<N> s(op, (size_t)idx[0], (size_t)idx[1], (size_t)idx[2], (size_t)idx[3], symm != 0);
        if (add) s.perform(bt, d);
        else s.perform(bt);
    }
};

template<size_t N>
void symmetrize_op(additive_gen_bto<N, btod_traits::bti_traits> &op, int nidx, const int32_t *idx, int symm,
    void *b, int add, double d) {
    symm_impl<N>::run(op, nidx, idx, symm, b, add, d);
}

template<size_t N>
void symmetrize_copy(void *a, double c, int nidx, const int32_t *idx, int symm, void *b, int add, double d) {
    btod_copy<N> cp(as<N>(a)->bt, c);
    symmetrize_op<N>(cp, nidx, idx, symm, b, add, d);
}

/* ---------------- contraction ------------------------------------------ */

struct c2_base {
    virtual ~c2_base() {}
    virtual size_t schedule(int64_t *out, size_t cap) = 0;
    virtual void *make_result() = 0;
    virtual void perform(void *c, int add, double d) = 0;
    virtual size_t clst(int64_t cabs, int64_t *out, size_t cap) = 0;
    virtual void cost(int64_t *exact, int64_t *ref_cost) = 0;
    virtual void symmetrize(int nidx, const int32_t *idx, int symm, void *b, int add, double d) = 0;
    virtual void result_bidims(int64_t *out) = 0;
};

template<size_t N, size_t M, size_t K>
struct c2_h : c2_base {
    enum { NA = N + K, NB = M + K, NC = N + M };
    contraction2<N, M, K> contr;
    bt_h<NA> *a; bt_h<NB> *b;
    btod_contract2<N, M, K> op;

    c2_h(const contraction2<N, M, K> &c, bt_h<NA> *a_, double ka,
         bt_h<NB> *b_, double kb, double kc) :
        contr(c), a(a_), b(b_), op(c, a_->bt, ka, b_->bt, kb, kc) {}

    size_t schedule(int64_t *out, size_t cap) {
        const assignment_schedule<NC, double> &sch = op.get_schedule();
        size_t i = 0;
        for (typename assignment_schedule<NC, double>::iterator it = sch.begin();
             it != sch.end(); ++it, ++i) {
            if (i < cap) out[i] = (int64_t)sch.get_abs_index(it);
        }
        return i;
    }

    void symmetrize(int nidx, const int32_t *idx, int symm, void *b, int add, double d) {
        symmetrize_op<NC>(op, nidx, idx, symm, b, add, d);
    }

    void *make_result() {
        bt_h<NC> *c = new bt_h<NC>(op.get_bis());
        block_tensor_wr_ctrl<NC, double> ctrl(c->bt);
        so_copy<NC, double>(op.get_symmetry()).perform(ctrl.req_symmetry());
        return c;
    }

    void result_bidims(int64_t *out) {
        dimensions<NC> bd = op.get_bis().get_block_index_dims();
        for (size_t d = 0; d < NC; d++) out[d] = (int64_t)bd[d];
    }

    void perform(void *c, int add, double d) {
        bt_h<NC> *ch = as<NC>(c);
        if (add) op.perform(ch->bt, d);
        else op.perform(ch->bt);
    }

    /* Unfolded non-zero block lists of A and B and the contraction block
       list built from them: the inputs of every per-C-block pair list
       (gen_bto_contract2_nzorb_impl.h:354-463).  Built on first use and kept,
       so that pair lists of many C blocks cost one list build each. */
    struct lists {
        block_list<NA> blax;
        block_list<NB> blbx;
        std::unique_ptr< gen_bto_contract2_block_list<N, M, K> > cbl;
        lists(const dimensions<NA> &da, const dimensions<NB> &db) :
            blax(da), blbx(db) {}
    };
    std::unique_ptr<lists> m_lists;

    lists &get_lists() {
        if (m_lists) return *m_lists;
        gen_block_tensor_rd_ctrl<NA, block_tensor_i_traits<double> > ca(a->bt);
        gen_block_tensor_rd_ctrl<NB, block_tensor_i_traits<double> > cb(b->bt);
        dimensions<NA> bidimsa = a->bis.get_block_index_dims();
        dimensions<NB> bidimsb = b->bis.get_block_index_dims();
        std::unique_ptr<lists> l(new lists(bidimsa, bidimsb));
        std::vector<size_t> v;
        block_list<NA> bla(bidimsa);
        block_list<NB> blb(bidimsb);
        ca.req_nonzero_blocks(v);
        for (size_t i = 0; i < v.size(); i++) bla.add(v[i]);
        cb.req_nonzero_blocks(v);
        for (size_t i = 0; i < v.size(); i++) blb.add(v[i]);
        gen_bto_unfold_block_list<NA, btod_traits>(ca.req_const_symmetry(), bla).build(l->blax);
        gen_bto_unfold_block_list<NB, btod_traits>(cb.req_const_symmetry(), blb).build(l->blbx);
        l->cbl.reset(new gen_bto_contract2_block_list<N, M, K>(contr, bidimsa,
            l->blax, bidimsb, l->blbx));
        m_lists = std::move(l);
        return *m_lists;
    }

    /* Pair list of one C block: the same call sequence the schedule builder
       makes (gen_bto_contract2_nzorb_impl.h:354-463).  Output per pair:
       aia, acia, perm_a[NA], coeff_a, aib, acib, perm_b[NB], coeff_b
       (coefficients as int64 of 1e6 * value is lossy, so they are returned
       as raw IEEE bits). */
    size_t clst(int64_t cabs, int64_t *out, size_t cap) {
        gen_block_tensor_rd_ctrl<NA, block_tensor_i_traits<double> > ca(a->bt);
        gen_block_tensor_rd_ctrl<NB, block_tensor_i_traits<double> > cb(b->bt);
        const symmetry<NA, double> &syma = ca.req_const_symmetry();
        const symmetry<NB, double> &symb = cb.req_const_symmetry();
        dimensions<NC> bidimsc = op.get_bis().get_block_index_dims();
        lists &l = get_lists();
        index<NC> ic;
        abs_index<NC>::get_index((size_t)cabs, bidimsc, ic);
        gen_bto_contract2_clst_builder<N, M, K, btod_traits> bld(contr, syma,
            symb, l.blax, l.blbx, bidimsc, ic);
        bld.build_list(false, *l.cbl);
        const typename gen_bto_contract2_clst<N, M, K, double>::list_type &lst =
            bld.get_clst();
        size_t rec = 2 + NA + 1 + 2 + NB + 1, k = 0;
        for (typename gen_bto_contract2_clst<N, M, K, double>::list_type::
                const_iterator it = lst.begin(); it != lst.end(); ++it, ++k) {
            if ((k + 1) * rec > cap) continue;
            int64_t *o = out + k * rec;
            o[0] = (int64_t)it->get_aindex_a();
            o[1] = (int64_t)it->get_acindex_a();
            for (size_t d = 0; d < NA; d++)
                o[2 + d] = (int64_t)it->get_transf_a().get_perm()[d];
            double ca_ = it->get_transf_a().get_scalar_tr().get_coeff();
            std::memcpy(&o[2 + NA], &ca_, 8);
            int64_t *q = o + 3 + NA;
            q[0] = (int64_t)it->get_aindex_b();
            q[1] = (int64_t)it->get_acindex_b();
            for (size_t d = 0; d < NB; d++)
                q[2 + d] = (int64_t)it->get_transf_b().get_perm()[d];
            double cb_ = it->get_transf_b().get_scalar_tr().get_coeff();
            std::memcpy(&q[2 + NB], &cb_, 8);
        }
        return k;
    }

    /* Work of the whole schedule as the reference's task cost counts it
       (gen_bto_contract2_block_impl.h:63-95, applied to the coalesced pair
       list of every scheduled C block): per pair, the product of A's block
       extents on the indices contracted with B, times the C block's size.
       exact = that sum without the reference's per-pair integer division by
       1000; ref_cost = the sum of the reference's own per-pair summands. */
    void cost(int64_t *exact, int64_t *ref_cost) {
        gen_block_tensor_rd_ctrl<NA, block_tensor_i_traits<double> > ca(a->bt);
        gen_block_tensor_rd_ctrl<NB, block_tensor_i_traits<double> > cb(b->bt);
        const symmetry<NA, double> &syma = ca.req_const_symmetry();
        const symmetry<NB, double> &symb = cb.req_const_symmetry();
        const block_index_space<NC> &bisc = op.get_bis();
        dimensions<NC> bidimsc = bisc.get_block_index_dims();
        dimensions<NA> bidimsa = a->bis.get_block_index_dims();
        const sequence<NA + NB + NC, size_t> &conn = contr.get_conn();
        lists &l = get_lists();
        const assignment_schedule<NC, double> &sch = op.get_schedule();
        int64_t ex = 0, rc = 0;
        for (typename assignment_schedule<NC, double>::iterator it = sch.begin();
             it != sch.end(); ++it) {
            index<NC> ic;
            abs_index<NC>::get_index(sch.get_abs_index(it), bidimsc, ic);
            gen_bto_contract2_clst_builder<N, M, K, btod_traits> bld(contr,
                syma, symb, l.blax, l.blbx, bidimsc, ic);
            bld.build_list(false, *l.cbl);
            size_t szc = bisc.get_block_dims(ic).get_size();
            const typename gen_bto_contract2_clst<N, M, K, double>::list_type
                &lst = bld.get_clst();
            for (typename gen_bto_contract2_clst<N, M, K, double>::list_type::
                    const_iterator p = lst.begin(); p != lst.end(); ++p) {
                index<NA> ia;
                abs_index<NA>::get_index(p->get_aindex_a(), bidimsa, ia);
                dimensions<NA> dimsa = a->bis.get_block_dims(ia);
                size_t c = 1;
                for (size_t j = 0; j < NA; j++)
                    if (conn[NC + j] >= NA + NC) c *= dimsa[j];
                ex += (int64_t)(c * szc);
                rc += (int64_t)(c * szc / 1000);
            }
        }
        *exact = ex;
        *ref_cost = rc;
    }
};

template<size_t N, size_t M, size_t K>
c2_base *make_c2(const int32_t *permc, const int32_t *pairs, void *a,
    double ka, void *b, double kb, double kc) {
    contraction2<N, M, K> c(perm_from<N + M>(permc));
    for (size_t k = 0; k < K; k++) c.contract((size_t)pairs[2 * k], (size_t)pairs[2 * k + 1]);
    return new c2_h<N, M, K>(c, as<N + K>(a), ka, as<M + K>(b), kb, kc);
}

/* ---------------- copy / add / dotprod --------------------------------- */

template<size_t N>
void do_copy(void *a, const int32_t *perm, double c, void *b, int add, double d) {
    btod_copy<N> op(as<N>(a)->bt, perm_from<N>(perm), c);
    if (add) op.perform(as<N>(b)->bt, d);
    else op.perform(as<N>(b)->bt);
}

template<size_t N>
void do_add(int nt, void **as_, const int32_t *perms, const double *cs,
    void *b, int add, double d) {
    btod_add<N> op(as<N>(as_[0])->bt, perm_from<N>(perms), cs[0]);
    for (int t = 1; t < nt; t++)
        op.add_op(as<N>(as_[t])->bt, perm_from<N>(perms + t * N), cs[t]);
    if (add) op.perform(as<N>(b)->bt, d);
    else op.perform(as<N>(b)->bt);
}

template<size_t N>
double do_dot(void *a, const int32_t *pa, void *b, const int32_t *pb) {
    btod_dotprod<N> op(as<N>(a)->bt, perm_from<N>(pa), as<N>(b)->bt,
        perm_from<N>(pb));
    return op.calculate();
}

#define DISPATCH_ORDER(n, call) \
    switch (n) { \
    case 1: call(1); break; case 2: call(2); break; case 3: call(3); break; \
    case 4: call(4); break; case 5: call(5); break; case 6: call(6); break; \
    default: throw std::runtime_error("unsupported tensor order"); }

} // namespace

extern "C" {

const char *ref_last_error() { return g_err.c_str(); }

/* Associates a thread pool of nthreads workers with the calling thread and
   pins OpenBLAS to one thread, as the reference's own test drivers do
   (tests/block_tensor/libtensor_block_tensor_tests.C:64-65). */
int ref_set_threads(int nthreads) {
    try {
        openblas_set_num_threads(1);
        if (g_pool) { g_pool->dissociate(); g_pool->terminate(); g_pool.reset(); }
        if (nthreads > 1) {
            g_pool.reset(new libutil::thread_pool(nthreads, nthreads));
            g_pool->associate();
        }
        return 0;
    } catch (std::exception &e) { g_err = e.what(); return -1; }
}

void ref_set_batch_size(int64_t b) { batching_policy_base::set_batch_size((size_t)b); }

void *ref_bt_create(const int64_t *spec, int64_t n) {
    try {
        spec_reader r{spec, (size_t)n, 0};
        int64_t order = r.next();
        void *h = 0;
#define MK(k) h = make_bt<k>(r)
        DISPATCH_ORDER(order, MK)
#undef MK
        return h;
    } catch (libtensor::exception &e) { g_err = e.what(); return 0; }
    catch (std::exception &e) { g_err = e.what(); return 0; }
}

void ref_bt_destroy(void *h) { delete static_cast<bt_base*>(h); }

int ref_bt_order(void *h) { return (int)static_cast<bt_base*>(h)->order; }

int ref_bt_set_block(void *h, const int64_t *bidx, const double *data, int64_t n) {
    try {
        int r = 0;
#define CALL(k) r = set_block<k>(h, bidx, data, (size_t)n)
        DISPATCH_ORDER(static_cast<bt_base*>(h)->order, CALL)
#undef CALL
        return r;
    } catch (libtensor::exception &e) { g_err = e.what(); return -1; }
    catch (std::exception &e) { g_err = e.what(); return -1; }
}

int ref_bt_get_block(void *h, const int64_t *bidx, double *data, int64_t n) {
    try {
        int r = 0;
#define CALL(k) r = get_block<k>(h, bidx, data, (size_t)n)
        DISPATCH_ORDER(static_cast<bt_base*>(h)->order, CALL)
#undef CALL
        return r;
    } catch (libtensor::exception &e) { g_err = e.what(); return -1; }
    catch (std::exception &e) { g_err = e.what(); return -1; }
}

int64_t ref_bt_nonzero(void *h, int64_t *out, int64_t cap) {
    try {
        size_t r = 0;
#define CALL(k) r = nonzero<k>(h, out, (size_t)cap)
        DISPATCH_ORDER(static_cast<bt_base*>(h)->order, CALL)
#undef CALL
        return (int64_t)r;
    } catch (libtensor::exception &e) { g_err = e.what(); return -1; }
    catch (std::exception &e) { g_err = e.what(); return -1; }
}

int ref_bt_block_index_dims(void *h, int64_t *out) {
    try {
#define CALL(k) block_index_dims<k>(h, out)
        DISPATCH_ORDER(static_cast<bt_base*>(h)->order, CALL)
#undef CALL
        return 0;
    } catch (std::exception &e) { g_err = e.what(); return -1; }
}

/* Orbit of block aidx: canonical abs index, transform canonical -> aidx,
   orbit size; returns 1 if allowed, 0 if forbidden, -1 on error
   (core/impl/orbit_impl.h:139-297). */
int ref_bt_orbit(void *h, int64_t aidx, int64_t *canon, int32_t *perm,
    double *coeff, int64_t *orbit_size) {
    try {
        int r = 0;
#define CALL(k) r = orbit_info<k>(h, aidx, canon, perm, coeff, orbit_size)
        DISPATCH_ORDER(static_cast<bt_base*>(h)->order, CALL)
#undef CALL
        return r;
    } catch (libtensor::exception &e) { g_err = e.what(); return -1; }
    catch (std::exception &e) { g_err = e.what(); return -1; }
}

/* Seeded test inputs in the reference tensor (see fill_seeded): the group
   elements (perm[N] and sign per element, the full closure of the tensor's
   se_perm generators) are passed by the caller. */
int ref_bt_fill_seeded(void *h, uint64_t seed, double scale, int ngroup,
    const int32_t *perms, const int32_t *signs, int nthreads) {
    try {
#define CALL(k) fill_seeded<k>(h, seed, scale, ngroup, perms, signs, nthreads)
        DISPATCH_ORDER(static_cast<bt_base*>(h)->order, CALL)
#undef CALL
        return 0;
    } catch (libtensor::exception &e) { g_err = e.what(); return -1; }
    catch (std::exception &e) { g_err = e.what(); return -1; }
}

int ref_denominator(void *h, const double *eps, int nocc) {
    try {
#define CALL(k) denominator<k>(h, eps, nocc)
        DISPATCH_ORDER(static_cast<bt_base*>(h)->order, CALL)
#undef CALL
        return 0;
    } catch (libtensor::exception &e) { g_err = e.what(); return -1; }
    catch (std::exception &e) { g_err = e.what(); return -1; }
}

void *ref_contract2_create(int n, int m, int k, const int32_t *permc,
    const int32_t *pairs, void *a, double ka, void *b, double kb, double kc) {
    try {
        int key = n * 100 + m * 10 + k;
        switch (key) {
#define C2(N_, M_, K_) case N_ * 100 + M_ * 10 + K_: \
            return make_c2<N_, M_, K_>(permc, pairs, a, ka, b, kb, kc);
        C2(1, 1, 1) C2(1, 1, 2) C2(2, 1, 1) C2(1, 2, 1) C2(2, 2, 1)
        C2(2, 2, 2) C2(1, 3, 1) C2(3, 1, 1) C2(2, 1, 2) C2(1, 2, 2)
        C2(2, 2, 0) C2(1, 1, 0) C2(0, 2, 2) C2(2, 0, 2) C2(1, 1, 3)
#undef C2
        default: throw std::runtime_error("unsupported (N,M,K)");
        }
    } catch (libtensor::exception &e) { g_err = e.what(); return 0; }
    catch (std::exception &e) { g_err = e.what(); return 0; }
}

void ref_contract2_destroy(void *op) { delete static_cast<c2_base*>(op); }

int64_t ref_contract2_schedule(void *op, int64_t *out, int64_t cap) {
    try { return (int64_t)static_cast<c2_base*>(op)->schedule(out, (size_t)cap); }
    catch (libtensor::exception &e) { g_err = e.what(); return -1; }
    catch (std::exception &e) { g_err = e.what(); return -1; }
}

void *ref_contract2_make_result(void *op) {
    try { return static_cast<c2_base*>(op)->make_result(); }
    catch (libtensor::exception &e) { g_err = e.what(); return 0; }
    catch (std::exception &e) { g_err = e.what(); return 0; }
}

int ref_contract2_result_bidims(void *op, int64_t *out) {
    try { static_cast<c2_base*>(op)->result_bidims(out); return 0; }
    catch (std::exception &e) { g_err = e.what(); return -1; }
}

int ref_contract2_perform(void *op, void *c, int add, double d) {
    try { static_cast<c2_base*>(op)->perform(c, add, d); return 0; }
    catch (libtensor::exception &e) { g_err = e.what(); return -1; }
    catch (std::exception &e) { g_err = e.what(); return -1; }
}

int64_t ref_contract2_clst(void *op, int64_t cabs, int64_t *out, int64_t cap) {
    try { return (int64_t)static_cast<c2_base*>(op)->clst(cabs, out, (size_t)cap); }
    catch (libtensor::exception &e) { g_err = e.what(); return -1; }
    catch (std::exception &e) { g_err = e.what(); return -1; }
}

/* Work of the schedule as the reference's task cost counts it; see
   c2_h::cost. */
int ref_contract2_cost(void *op, int64_t *exact, int64_t *ref_cost) {
    try { static_cast<c2_base*>(op)->cost(exact, ref_cost); return 0; }
    catch (libtensor::exception &e) { g_err = e.what(); return -1; }
    catch (std::exception &e) { g_err = e.what(); return -1; }
}

/* Symmetrizer of a tensor (wrapping btod_copy with coefficient c) or of a
   contraction.  nidx 2: indexes idx[0], idx[1]; -1: the unitary permutation
   idx[0..N); 4: the four indexes idx[0..3]. */
int ref_symmetrize(void *a, double c, int nidx, const int32_t *idx, int symm, void *b, int add, double d) {
    try {
#define CALL(k) symmetrize_copy<k>(a, c, nidx, idx, symm, b, add, d)
        DISPATCH_ORDER(static_cast<bt_base*>(a)->order, CALL)
#undef CALL
        return 0;
    } catch (libtensor::exception &e) { g_err = e.what(); return -1; }
    catch (std::exception &e) { g_err = e.what(); return -1; }
}

int ref_contract2_symmetrize(void *op, int nidx, const int32_t *idx, int symm, void *b, int add, double d) {
    try { static_cast<c2_base*>(op)->symmetrize(nidx, idx, symm, b, add, d); return 0; }
    catch (libtensor::exception &e) { g_err = e.what(); return -1; }
    catch (std::exception &e) { g_err = e.what(); return -1; }
}

int ref_copy(void *a, const int32_t *perm, double c, void *b, int add, double d) {
    try {
#define CALL(k) do_copy<k>(a, perm, c, b, add, d)
        DISPATCH_ORDER(static_cast<bt_base*>(a)->order, CALL)
#undef CALL
        return 0;
    } catch (libtensor::exception &e) { g_err = e.what(); return -1; }
    catch (std::exception &e) { g_err = e.what(); return -1; }
}

int ref_add(int nterms, void **as_, const int32_t *perms, const double *coeffs,
    void *b, int add, double d) {
    try {
#define CALL(k) do_add<k>(nterms, as_, perms, coeffs, b, add, d)
        DISPATCH_ORDER(static_cast<bt_base*>(b)->order, CALL)
#undef CALL
        return 0;
    } catch (libtensor::exception &e) { g_err = e.what(); return -1; }
    catch (std::exception &e) { g_err = e.what(); return -1; }
}

int ref_dotprod(void *a, const int32_t *pa, void *b, const int32_t *pb, double *out) {
    try {
#define CALL(k) *out = do_dot<k>(a, pa, b, pb)
        DISPATCH_ORDER(static_cast<bt_base*>(a)->order, CALL)
#undef CALL
        return 0;
    } catch (libtensor::exception &e) { g_err = e.what(); return -1; }
    catch (std::exception &e) { g_err = e.what(); return -1; }
}

} // extern "C"
