/*
 * libtensor_b200/libtensor.h -- C++ operator surface of the B200 block-tensor
 * contraction path, over the C ABI of ltg.h.
 *
 * Mirrors the class templates a libtensor user writes against for this path,
 * in namespace libtensor, with the same names, argument meaning and error
 * behaviour (exceptions of the same names):
 *   index, index_range, dimensions, mask, permutation, scalar_transf,
 *   block_index_space (libtensor/core/block_index_space.h:144),
 *   se_perm (libtensor/symmetry/se_perm.h:28), se_part (se_part.h:32),
 *   se_label (se_label.h:37) for abelian point groups, symmetry,
 *   block_tensor and block_tensor_ctrl (libtensor/block_tensor/block_tensor.h:22),
 *   contraction2 (libtensor/core/contraction2.h:48),
 *   btod_contract2 (libtensor/block_tensor/btod_contract2.h:29),
 *   btod_copy (btod_copy.h:38), btod_add (btod_add.h:38),
 *   btod_dotprod (btod_dotprod.h:35),
 *   and the letter interface over them (libtensor/expr/iface/letter.h,
 *   label.h, expr_rhs.h; operators/contract.h, plus_minus.h,
 *   multiply_divide.h, dot_product.h): letter, label, operator|, btensor,
 *   t(i|j|a|b) = expression, +=, -=, contract, dot_product.
 * Differences a user meets:
 *   - block data lives in GPU memory; blocks are read and written with
 *     block_tensor_ctrl::get_block / put_block (host buffers) instead of the
 *     dense_tensor_ctrl data-pointer sessions;
 *   - symmetry elements are inserted before the first data access or
 *     operation (the device layout is built from them);
 *   - se_label supports abelian (XOR) product tables of 1, 2, 4 or 8
 *     irreducible representations, registered by name with
 *     register_abelian_table();
 *   - btod_contract2::set_split_precision() selects the split-precision
 *     modes of ltg.h (the default is the FP64 drop-in path).
 * Header-only; link with libltg.so.
 */
#ifndef LIBTENSOR_B200_LIBTENSOR_H
#define LIBTENSOR_B200_LIBTENSOR_H

#include <array>
#include <functional>
#include <initializer_list>
#include <cstddef>
#include <cstdint>
#include <map>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../ltg.h"

namespace libtensor {

// ---------------------------------------------------------------- exceptions

class exception : public std::runtime_error {
public:
    explicit exception(const std::string &what) : std::runtime_error(what) { }
};
class bad_parameter : public exception { public: using exception::exception; };
class bad_dimensions : public exception { public: using exception::exception; };
class bad_symmetry : public exception { public: using exception::exception; };
class out_of_bounds : public exception { public: using exception::exception; };
class device_error : public exception { public: using exception::exception; };

namespace b200 {

// Converts an ltg status into the exception class of the reference.
inline void check(int st) {
    if (st == LTG_OK) return;
    const std::string msg = ltg_last_error();
    switch (st) {
    case LTG_ERR_BAD_DIMS: throw bad_dimensions(msg);
    case LTG_ERR_SYMMETRY: throw bad_symmetry(msg);
    case LTG_ERR_BAD_ARG: throw bad_parameter(msg);
    default: throw device_error(msg);
    }
}

// The process-wide context of the surface: device 0 unless set_device() is
// called before the first block tensor is used (device -1: host only, for
// schedules and symmetry queries without a GPU).
struct context_holder {
    int device = 0;
    ltg_ctx *ctx = nullptr;
    ~context_holder() { if (ctx) ltg_ctx_destroy(ctx); }
};
inline context_holder &holder() {
    static context_holder h;
    return h;
}
inline void set_device(int device) {
    if (holder().ctx) throw bad_parameter("set_device: the context is already in use");
    holder().device = device;
}
inline ltg_ctx *context() {
    context_holder &h = holder();
    if (!h.ctx) check(ltg_ctx_create(h.device, &h.ctx));
    return h.ctx;
}

// Abelian product tables for se_label, by name: XOR of irrep indices.
inline std::map<std::string, int> &abelian_tables() {
    static std::map<std::string, int> t;
    return t;
}
}  // namespace b200

// Registers an abelian point-group product table (irreps combine by XOR of
// their indices, as in D2h and its subgroups) under a name for se_label.
inline void register_abelian_table(const std::string &id, int nirrep) {
    if (nirrep != 1 && nirrep != 2 && nirrep != 4 && nirrep != 8)
        throw bad_parameter("register_abelian_table: 1, 2, 4 or 8 irreps");
    b200::abelian_tables()[id] = nirrep;
}

// ---------------------------------------------------------------- index types

template<size_t N>
class index {
    size_t m_i[N == 0 ? 1 : N];
public:
    index() { for (size_t i = 0; i < N; i++) m_i[i] = 0; }
    size_t &operator[](size_t i) { return m_i[i]; }
    const size_t &operator[](size_t i) const { return m_i[i]; }
    size_t at(size_t i) const { if (i >= N) throw out_of_bounds("index::at"); return m_i[i]; }
    bool equals(const index<N> &o) const {
        for (size_t i = 0; i < N; i++) if (m_i[i] != o.m_i[i]) return false;
        return true;
    }
    bool operator==(const index<N> &o) const { return equals(o); }
    bool operator<(const index<N> &o) const {
        for (size_t i = 0; i < N; i++) if (m_i[i] != o.m_i[i]) return m_i[i] < o.m_i[i];
        return false;
    }
};

template<size_t N>
class index_range {
    index<N> m_begin, m_end;
public:
    index_range(const index<N> &begin, const index<N> &end) : m_begin(begin), m_end(end) {
        for (size_t i = 0; i < N; i++)
            if (end[i] < begin[i]) throw bad_parameter("index_range: end before begin");
    }
    const index<N> &get_begin() const { return m_begin; }
    const index<N> &get_end() const { return m_end; }
};

template<size_t N>
class dimensions {
    index<N> m_d;
public:
    explicit dimensions(const index_range<N> &ir) {
        for (size_t i = 0; i < N; i++) m_d[i] = ir.get_end()[i] - ir.get_begin()[i] + 1;
    }
    size_t get_dim(size_t i) const { return m_d.at(i); }
    size_t operator[](size_t i) const { return m_d[i]; }
    size_t get_size() const {
        size_t n = 1;
        for (size_t i = 0; i < N; i++) n *= m_d[i];
        return n;
    }
    bool equals(const dimensions<N> &o) const { return m_d.equals(o.m_d); }
};

template<size_t N>
class mask {
    bool m_m[N == 0 ? 1 : N];
public:
    mask() { for (size_t i = 0; i < N; i++) m_m[i] = false; }
    bool &operator[](size_t i) { return m_m[i]; }
    bool operator[](size_t i) const { return m_m[i]; }
};

// permutation<N>: element i of a permuted sequence is element p[i] of the
// original (libtensor/core/permutation.h).
template<size_t N>
class permutation {
    size_t m_p[N == 0 ? 1 : N];
public:
    permutation() { for (size_t i = 0; i < N; i++) m_p[i] = i; }
    // from the sequence p[0..N) (a permutation of 0..N-1)
    explicit permutation(const std::vector<size_t> &p) {
        if (p.size() != N) throw bad_parameter("permutation: wrong length");
        std::vector<char> seen(N, 0);
        for (size_t i = 0; i < N; i++) {
            if (p[i] >= N || seen[p[i]]) throw bad_parameter("permutation: not a permutation");
            seen[p[i]] = 1;
            m_p[i] = p[i];
        }
    }
    permutation<N> &permute(size_t i, size_t j) {
        if (i >= N || j >= N) throw out_of_bounds("permutation::permute");
        std::swap(m_p[i], m_p[j]);
        return *this;
    }
    permutation<N> &permute(const permutation<N> &q) {
        size_t r[N == 0 ? 1 : N];
        for (size_t i = 0; i < N; i++) r[i] = m_p[q.m_p[i]];
        for (size_t i = 0; i < N; i++) m_p[i] = r[i];
        return *this;
    }
    permutation<N> &invert() {
        size_t r[N == 0 ? 1 : N];
        for (size_t i = 0; i < N; i++) r[m_p[i]] = i;
        for (size_t i = 0; i < N; i++) m_p[i] = r[i];
        return *this;
    }
    bool is_identity() const {
        for (size_t i = 0; i < N; i++) if (m_p[i] != i) return false;
        return true;
    }
    size_t operator[](size_t i) const { return m_p[i]; }
    std::vector<int32_t> to_vector() const { return std::vector<int32_t>(m_p, m_p + N); }
};

template<typename T>
class scalar_transf {
    T m_c;
public:
    explicit scalar_transf(T c = T(1)) : m_c(c) { }
    T get_coeff() const { return m_c; }
};

// ---------------------------------------------------------------- block index space

template<size_t N>
class block_index_space {
    dimensions<N> m_dims;
    std::vector<size_t> m_splits[N == 0 ? 1 : N];
public:
    explicit block_index_space(const dimensions<N> &dims) : m_dims(dims) { }
    const dimensions<N> &get_dims() const { return m_dims; }
    // splits every dim set in msk at position pos
    void split(const mask<N> &msk, size_t pos) {
        for (size_t i = 0; i < N; i++) {
            if (!msk[i]) continue;
            if (pos == 0 || pos >= m_dims[i]) throw out_of_bounds("block_index_space::split");
            std::vector<size_t> &s = m_splits[i];
            std::vector<size_t>::iterator it = s.begin();
            while (it != s.end() && *it < pos) ++it;
            if (it == s.end() || *it != pos) s.insert(it, pos);
        }
    }
    const std::vector<size_t> &get_splits(size_t dim) const { return m_splits[dim]; }
    dimensions<N> get_block_index_dims() const {
        index<N> i1;
        for (size_t i = 0; i < N; i++) i1[i] = m_splits[i].size();
        return dimensions<N>(index_range<N>(index<N>(), i1));
    }
    index<N> get_block_start(const index<N> &bidx) const {
        index<N> s;
        for (size_t i = 0; i < N; i++) s[i] = bidx[i] == 0 ? 0 : m_splits[i].at(bidx[i] - 1);
        return s;
    }
    dimensions<N> get_block_dims(const index<N> &bidx) const {
        index<N> i1;
        for (size_t i = 0; i < N; i++) {
            const size_t b0 = bidx[i] == 0 ? 0 : m_splits[i].at(bidx[i] - 1);
            const size_t b1 = bidx[i] < m_splits[i].size() ? m_splits[i][bidx[i]] : m_dims[i];
            i1[i] = b1 - b0 - 1;
        }
        return dimensions<N>(index_range<N>(index<N>(), i1));
    }
    bool equals(const block_index_space<N> &o) const {
        if (!m_dims.equals(o.m_dims)) return false;
        for (size_t i = 0; i < N; i++) if (m_splits[i] != o.m_splits[i]) return false;
        return true;
    }
};

// ---------------------------------------------------------------- symmetry elements

template<size_t N, typename T>
class se_perm {
    permutation<N> m_perm;
    scalar_transf<T> m_tr;
public:
    se_perm(const permutation<N> &perm, const scalar_transf<T> &tr) : m_perm(perm), m_tr(tr) {
        if (perm.is_identity() && tr.get_coeff() != T(1))
            throw bad_symmetry("se_perm: identity permutation with a non-unit coefficient");
    }
    const permutation<N> &get_perm() const { return m_perm; }
    const scalar_transf<T> &get_transf() const { return m_tr; }
};

// Partitions of block dims with forbidden partition combinations (the
// partition maps of the reference's se_part are not supported).
template<size_t N, typename T>
class se_part {
    index<N> m_pdims;
    std::vector<index<N> > m_forbidden;
public:
    se_part(const block_index_space<N> &bis, const mask<N> &msk, size_t npart) {
        const dimensions<N> bd = bis.get_block_index_dims();
        for (size_t i = 0; i < N; i++) {
            m_pdims[i] = msk[i] ? npart : 1;
            if (msk[i] && (npart == 0 || bd[i] % npart != 0))
                throw bad_parameter("se_part: partitions must divide the number of blocks");
        }
    }
    se_part(const block_index_space<N> &bis, const dimensions<N> &pdims) {
        const dimensions<N> bd = bis.get_block_index_dims();
        for (size_t i = 0; i < N; i++) {
            m_pdims[i] = pdims[i];
            if (pdims[i] == 0 || bd[i] % pdims[i] != 0)
                throw bad_parameter("se_part: partitions must divide the number of blocks");
        }
    }
    void mark_forbidden(const index<N> &pidx) {
        for (size_t i = 0; i < N; i++)
            if (pidx[i] >= m_pdims[i]) throw out_of_bounds("se_part::mark_forbidden");
        m_forbidden.push_back(pidx);
    }
    const index<N> &get_pdims() const { return m_pdims; }
    const std::vector<index<N> > &get_forbidden() const { return m_forbidden; }
};

typedef size_t label_t;

template<size_t N>
class block_labeling {
    std::vector<long> m_labels[N == 0 ? 1 : N];
public:
    explicit block_labeling(const dimensions<N> &bidims) {
        for (size_t i = 0; i < N; i++) m_labels[i].assign(bidims[i], -1);
    }
    // labels block blk of every dim set in msk
    void assign(const mask<N> &msk, size_t blk, label_t label) {
        for (size_t i = 0; i < N; i++)
            if (msk[i]) m_labels[i].at(blk) = (long)label;
    }
    const std::vector<long> &labels(size_t dim) const { return m_labels[dim]; }
};

template<size_t N, typename T>
class se_label {
    block_labeling<N> m_bl;
    int m_nirrep;
    std::set<label_t> m_rule;
public:
    se_label(const dimensions<N> &bidims, const std::string &id) : m_bl(bidims) {
        std::map<std::string, int>::const_iterator it = b200::abelian_tables().find(id);
        if (it == b200::abelian_tables().end())
            throw bad_parameter("se_label: product table '" + id + "' is not registered");
        m_nirrep = it->second;
    }
    block_labeling<N> &get_labeling() { return m_bl; }
    const block_labeling<N> &get_labeling() const { return m_bl; }
    void set_rule(label_t intr) { m_rule.clear(); m_rule.insert(intr); }
    void set_rule(const std::set<label_t> &intr) { m_rule = intr; }
    int get_nirrep() const { return m_nirrep; }
    const std::set<label_t> &get_rule() const { return m_rule; }
};

template<size_t N, typename T>
class symmetry {
    std::vector<se_perm<N, T> > m_perm;
    std::vector<se_part<N, T> > m_part;
    std::vector<se_label<N, T> > m_label;
public:
    void insert(const se_perm<N, T> &e) { m_perm.push_back(e); }
    void insert(const se_part<N, T> &e) {
        if (!m_part.empty()) throw bad_symmetry("symmetry: one se_part element is supported");
        m_part.push_back(e);
    }
    void insert(const se_label<N, T> &e) {
        if (!m_label.empty()) throw bad_symmetry("symmetry: one se_label element is supported");
        m_label.push_back(e);
    }
    void clear() { m_perm.clear(); m_part.clear(); m_label.clear(); }
    const std::vector<se_perm<N, T> > &perms() const { return m_perm; }
    const std::vector<se_part<N, T> > &parts() const { return m_part; }
    const std::vector<se_label<N, T> > &labels() const { return m_label; }
};

// ---------------------------------------------------------------- block tensor

template<size_t N, typename T> class block_tensor_ctrl;
template<size_t N> class label;
template<size_t N> class labeled_btensor;

template<size_t N, typename T>
class block_tensor {
    static_assert(sizeof(T) == 8, "block tensors of double");
    friend class block_tensor_ctrl<N, T>;
    block_index_space<N> m_bis;
    symmetry<N, T> m_sym;
    ltg_bt *m_bt = nullptr;
    block_tensor(const block_tensor &) = delete;
    block_tensor &operator=(const block_tensor &) = delete;
public:
    explicit block_tensor(const block_index_space<N> &bis) : m_bis(bis) { }
    virtual ~block_tensor() { if (m_bt) ltg_bt_destroy(m_bt); }
    const block_index_space<N> &get_bis() const { return m_bis; }
    bool is_bound() const { return m_bt != nullptr; }
    // The device tensor, built from the index space and symmetry on first use
    // (a direct block tensor first computes its operation's result).
    virtual ltg_bt *handle() {
        if (m_bt) return m_bt;
        std::vector<int64_t> dims(N), splits;
        std::vector<int32_t> nsplit(N), perm, labels, intr;
        std::vector<double> perm_coeff;
        std::vector<int64_t> pdims, forb;
        for (size_t i = 0; i < N; i++) {
            dims[i] = (int64_t)m_bis.get_dims()[i];
            nsplit[i] = (int32_t)m_bis.get_splits(i).size();
            for (size_t x : m_bis.get_splits(i)) splits.push_back((int64_t)x);
        }
        for (const se_perm<N, T> &e : m_sym.perms()) {
            for (size_t i = 0; i < N; i++) perm.push_back((int32_t)e.get_perm()[i]);
            perm_coeff.push_back((double)e.get_transf().get_coeff());
        }
        ltg_bt_spec s = {};
        s.order = (int32_t)N;
        s.dims = dims.data();
        s.nsplit = nsplit.data();
        s.splits = splits.data();
        s.nperm = (int32_t)m_sym.perms().size();
        s.perm = perm.data();
        s.perm_coeff = perm_coeff.data();
        if (!m_sym.parts().empty()) {
            const se_part<N, T> &p = m_sym.parts()[0];
            for (size_t i = 0; i < N; i++) pdims.push_back((int64_t)p.get_pdims()[i]);
            for (const index<N> &f : p.get_forbidden())
                for (size_t i = 0; i < N; i++) forb.push_back((int64_t)f[i]);
            s.has_part = 1;
            s.part_pdims = pdims.data();
            s.npart_forbidden = (int64_t)p.get_forbidden().size();
            s.part_forbidden = forb.data();
        }
        if (!m_sym.labels().empty()) {
            const se_label<N, T> &l = m_sym.labels()[0];
            for (size_t i = 0; i < N; i++)
                for (long v : l.get_labeling().labels(i)) labels.push_back((int32_t)v);
            for (label_t v : l.get_rule()) intr.push_back((int32_t)v);
            s.has_label = 1;
            s.label_nirrep = l.get_nirrep();
            s.labels = labels.data();
            s.label_nintr = (int32_t)intr.size();
            s.label_intr = intr.data();
        }
        b200::check(ltg_bt_create(b200::context(), &s, &m_bt));
        return m_bt;
    }
    // Adopts a device tensor with the same index space (results of operations).
    void adopt(ltg_bt *bt) {
        if (m_bt) ltg_bt_destroy(m_bt);
        m_bt = bt;
    }
    // t(i|j|a|b): the tensor labelled for the letter interface (defined below)
    template<size_t M> labeled_btensor<M> operator()(const label<M> &l);
};

template<size_t N, typename T>
class block_tensor_ctrl {
    block_tensor<N, T> &m_bt;
    static std::vector<int64_t> idx64(const index<N> &i) {
        std::vector<int64_t> v(N);
        for (size_t k = 0; k < N; k++) v[k] = (int64_t)i[k];
        return v;
    }
    std::vector<index<N> > unpack(const std::vector<int64_t> &abs) {
        std::vector<int64_t> bd(N);
        b200::check(ltg_bt_bidims(m_bt.handle(), bd.data()));
        std::vector<index<N> > out;
        for (int64_t a : abs) {
            index<N> i;
            for (size_t k = N; k-- > 0;) { i[k] = (size_t)(a % bd[k]); a /= bd[k]; }
            out.push_back(i);
        }
        return out;
    }
public:
    explicit block_tensor_ctrl(block_tensor<N, T> &bt) : m_bt(bt) { }
    symmetry<N, T> &req_symmetry() {
        if (m_bt.is_bound()) throw bad_symmetry("symmetry is fixed once the tensor holds data");
        return m_bt.m_sym;
    }
    const symmetry<N, T> &req_const_symmetry() const { return m_bt.m_sym; }
    // canonical, allowed block indices (the orbit list)
    std::vector<index<N> > req_canonical_blocks() {
        ltg_bt *h = m_bt.handle();
        int32_t order;
        int64_t nb, ne;
        b200::check(ltg_bt_info(h, &order, &nb, &ne));
        std::vector<int64_t> abs(nb > 0 ? nb : 1), off(abs.size()), sz(abs.size());
        b200::check(ltg_bt_blocks(h, abs.data(), off.data(), sz.data()));
        abs.resize(nb);
        return unpack(abs);
    }
    std::vector<index<N> > req_nonzero_blocks() {
        ltg_bt *h = m_bt.handle();
        int64_t n = 0;
        b200::check(ltg_bt_nonzero(h, nullptr, 0, &n));
        std::vector<int64_t> abs(n > 0 ? n : 1);
        b200::check(ltg_bt_nonzero(h, abs.data(), n, &n));
        abs.resize(n);
        return unpack(abs);
    }
    void put_block(const index<N> &bidx, const T *data) {
        b200::check(ltg_bt_upload_block(m_bt.handle(), idx64(bidx).data(), data));
    }
    void get_block(const index<N> &bidx, T *data) {
        b200::check(ltg_bt_download_block(m_bt.handle(), idx64(bidx).data(), data));
    }
    void req_zero_block(const index<N> &bidx) {
        b200::check(ltg_bt_zero_block(m_bt.handle(), idx64(bidx).data()));
    }
    void req_zero_all_blocks() { b200::check(ltg_bt_set_zero(m_bt.handle())); }
    // marks every canonical block non-zero without data (schedules on a
    // host-only context; not in the reference)
    void mark_nonzero() { b200::check(ltg_bt_mark_nonzero(m_bt.handle())); }
    // seeded test data (the product's generator; not in the reference)
    void fill_seeded(uint64_t seed, double scale) {
        b200::check(ltg_bt_fill_seeded(m_bt.handle(), seed, scale));
    }
};

// ---------------------------------------------------------------- contraction2

template<size_t N, size_t M, size_t K>
class contraction2 {
    permutation<N + M> m_permc;
    std::vector<std::pair<size_t, size_t> > m_pairs;
public:
    contraction2() { }
    explicit contraction2(const permutation<N + M> &permc) : m_permc(permc) { }
    bool is_complete() const { return m_pairs.size() == K; }
    void contract(size_t ia, size_t ib) {
        if (is_complete()) throw exception("contraction2::contract: contraction is complete");
        if (ia >= N + K || ib >= M + K) throw out_of_bounds("contraction2::contract");
        for (const std::pair<size_t, size_t> &p : m_pairs)
            if (p.first == ia || p.second == ib) throw bad_parameter("contraction2::contract: index used twice");
        m_pairs.push_back(std::make_pair(ia, ib));
    }
    const permutation<N + M> &get_permc() const { return m_permc; }
    const std::vector<std::pair<size_t, size_t> > &get_pairs() const { return m_pairs; }
};

// ---------------------------------------------------------------- operations

// An operation whose result can be assigned to or added into a block tensor
// (the role of libtensor's additive_gen_bto, gen_block_tensor/additive_gen_bto.h):
// what the symmetrizers wrap.
template<size_t N>
class additive_bto {
public:
    virtual ~additive_bto() { }
    virtual void perform(block_tensor<N, double> &btb) = 0;
    virtual void perform(block_tensor<N, double> &btb, double d) = 0;
    // btb = sum over the two-element symmetrizer group {e, P} of sign * P(this
    // operation's result), formed without the result itself where the
    // operation can (a plain FP64 contraction writes both terms from its
    // epilogue); false: not supported here, nothing done.
    virtual bool perform_symmetrized(block_tensor<N, double> &btb, int32_t nidx, const int32_t *idx, bool symm,
                                     ltg_bt **adopted) {
        (void)btb; (void)nidx; (void)idx; (void)symm; (void)adopted;
        return false;
    }
};

template<size_t N, size_t M, size_t K>
class btod_contract2 : public additive_bto<N + M> {
    ltg_plan *m_plan = nullptr;
    double m_ka, m_kb, m_kc;
    int32_t m_mode = LTG_MODE_PLAIN_FP64, m_nslices = 0;
    btod_contract2(const btod_contract2 &) = delete;
    btod_contract2 &operator=(const btod_contract2 &) = delete;
    void init(const contraction2<N, M, K> &contr, block_tensor<N + K, double> &bta,
              block_tensor<M + K, double> &btb) {
        if (!contr.is_complete()) throw bad_parameter("btod_contract2: incomplete contraction");
        std::vector<int32_t> permc = contr.get_permc().to_vector(), pairs;
        for (const std::pair<size_t, size_t> &p : contr.get_pairs()) {
            pairs.push_back((int32_t)p.first);
            pairs.push_back((int32_t)p.second);
        }
        b200::check(ltg_contract2_create(b200::context(), (int32_t)N, (int32_t)M, (int32_t)K, permc.data(),
                                         pairs.data(), bta.handle(), btb.handle(), &m_plan));
    }
    ltg_bt *m_adopted = nullptr;     // the result tensor the last assignment created
    void run(block_tensor<N + M, double> &btc, int32_t add, double d) {
        if (!add && !(btc.is_bound() && btc.handle() == m_adopted)) {
            // assignment gives C the result symmetry (as the reference's perform
            // does); repeated assignments to the same result reuse it, so
            // that they can be captured in a graph
            ltg_bt *c = nullptr;
            b200::check(ltg_contract2_make_result(m_plan, &c));
            btc.adopt(c);
            m_adopted = c;
        }
        b200::check(ltg_contract2(m_plan, btc.handle(), m_mode, m_nslices, m_ka, m_kb, m_kc, add, d));
    }
public:
    btod_contract2(const contraction2<N, M, K> &contr, block_tensor<N + K, double> &bta,
                   block_tensor<M + K, double> &btb) : m_ka(1.0), m_kb(1.0), m_kc(1.0) {
        init(contr, bta, btb);
    }
    btod_contract2(const contraction2<N, M, K> &contr, block_tensor<N + K, double> &bta, double ka,
                   block_tensor<M + K, double> &btb, double kb, double kc) : m_ka(ka), m_kb(kb), m_kc(kc) {
        init(contr, bta, btb);
    }
    ~btod_contract2() { if (m_plan) ltg_plan_destroy(m_plan); }
    // C = contraction (assign)
    void perform(block_tensor<N + M, double> &btc) override { run(btc, 0, 0.0); }
    // C += d * contraction
    void perform(block_tensor<N + M, double> &btc, double d) override { run(btc, 1, d); }
    void perform(block_tensor<N + M, double> &btc, const scalar_transf<double> &d) { run(btc, 1, d.get_coeff()); }
    // non-zero canonical result blocks (get_schedule), as absolute indices
    std::vector<int64_t> get_schedule() const {
        int64_t n = 0;
        b200::check(ltg_plan_schedule(m_plan, nullptr, 0, &n));
        std::vector<int64_t> v(n > 0 ? n : 1);
        b200::check(ltg_plan_schedule(m_plan, v.data(), n, &n));
        v.resize(n);
        return v;
    }
    double get_flops() const {
        double f = 0;
        b200::check(ltg_plan_flops(m_plan, &f));
        return f;
    }
    // LTG_MODE_OZAKI_* of ltg.h with its slice (or modulus) count; the
    // default LTG_MODE_PLAIN_FP64 is the FP64 drop-in path.
    void set_split_precision(int32_t mode, int32_t nslices) { m_mode = mode; m_nslices = nslices; }
    bool perform_symmetrized(block_tensor<N + M, double> &btb, int32_t nidx, const int32_t *idx, bool symm,
                             ltg_bt **adopted) override {
        if (nidx != 2 && nidx != -1) return false;
        if (!(btb.is_bound() && btb.handle() == *adopted)) {
            ltg_bt *r = nullptr;
            b200::check(ltg_contract2_make_symmetrized(m_plan, nidx, idx, symm ? 1 : 0, &r));
            btb.adopt(r);
            *adopted = r;
        }
        const int rc = ltg_contract2_symmetrized(m_plan, btb.handle(), m_mode, m_nslices, 1.0, nidx, idx,
                                                 symm ? 1 : 0, m_ka, m_kb, m_kc);
        if (rc == LTG_ERR_UNSUPPORTED) return false;   // e.g. too many destinations: through a temporary
        b200::check(rc);
        return true;
    }
};

template<size_t N>
class btod_copy : public additive_bto<N> {
    block_tensor<N, double> &m_a;
    permutation<N> m_perm;
    double m_c;
    ltg_bt *m_adopted = nullptr;     // as in btod_contract2
public:
    btod_copy(block_tensor<N, double> &bta, double c = 1.0) : m_a(bta), m_c(c) { }
    btod_copy(block_tensor<N, double> &bta, const permutation<N> &perm, double c = 1.0)
        : m_a(bta), m_perm(perm), m_c(c) { }
    // B = c P(A): B takes the permuted space and symmetry of A
    void perform(block_tensor<N, double> &btb) override {
        const std::vector<int32_t> p = m_perm.to_vector();
        if (!(btb.is_bound() && btb.handle() == m_adopted)) {
            ltg_bt *b = nullptr;
            b200::check(ltg_bt_create_permuted(m_a.handle(), p.data(), &b));
            btb.adopt(b);
            m_adopted = b;
        }
        b200::check(ltg_copy(m_a.handle(), p.data(), m_c, btb.handle(), 0, 0.0));
    }
    // B += d c P(A)
    void perform(block_tensor<N, double> &btb, double d) override {
        const std::vector<int32_t> p = m_perm.to_vector();
        b200::check(ltg_copy(m_a.handle(), p.data(), m_c, btb.handle(), 1, d));
    }
};

template<size_t N>
class btod_add : public additive_bto<N> {
    std::vector<block_tensor<N, double> *> m_ops;
    std::vector<permutation<N> > m_perms;
    std::vector<double> m_coeffs;
    void call(block_tensor<N, double> &btb, int32_t add, double d) {
        std::vector<ltg_bt *> hs;
        std::vector<int32_t> perms;
        for (size_t t = 0; t < m_ops.size(); t++) {
            hs.push_back(m_ops[t]->handle());
            const std::vector<int32_t> p = m_perms[t].to_vector();
            perms.insert(perms.end(), p.begin(), p.end());
        }
        b200::check(ltg_add((int32_t)hs.size(), hs.data(), perms.data(), m_coeffs.data(), btb.handle(), add, d));
    }
public:
    btod_add(block_tensor<N, double> &bt, double c = 1.0) { add_op(bt, c); }
    btod_add(block_tensor<N, double> &bt, const permutation<N> &perm, double c = 1.0) { add_op(bt, perm, c); }
    void add_op(block_tensor<N, double> &bt, double c = 1.0) { add_op(bt, permutation<N>(), c); }
    void add_op(block_tensor<N, double> &bt, const permutation<N> &perm, double c = 1.0) {
        m_ops.push_back(&bt);
        m_perms.push_back(perm);
        m_coeffs.push_back(c);
    }
    void perform(block_tensor<N, double> &btb) override { call(btb, 0, 0.0); }
    void perform(block_tensor<N, double> &btb, double d) override { call(btb, 1, d); }
};

template<size_t N>
class btod_dotprod {
    struct arg {
        block_tensor<N, double> *a, *b;
        permutation<N> pa, pb;
    };
    std::vector<arg> m_args;
public:
    btod_dotprod(block_tensor<N, double> &bt1, block_tensor<N, double> &bt2) { add_arg(bt1, bt2); }
    btod_dotprod(block_tensor<N, double> &bt1, const permutation<N> &perm1, block_tensor<N, double> &bt2,
                 const permutation<N> &perm2) { add_arg(bt1, perm1, bt2, perm2); }
    void add_arg(block_tensor<N, double> &bt1, block_tensor<N, double> &bt2) {
        add_arg(bt1, permutation<N>(), bt2, permutation<N>());
    }
    void add_arg(block_tensor<N, double> &bt1, const permutation<N> &perm1, block_tensor<N, double> &bt2,
                 const permutation<N> &perm2) {
        arg x;
        x.a = &bt1; x.b = &bt2; x.pa = perm1; x.pb = perm2;
        m_args.push_back(x);
    }
    void calculate(std::vector<double> &v) {
        v.resize(m_args.size());
        for (size_t i = 0; i < m_args.size(); i++) {
            const std::vector<int32_t> pa = m_args[i].pa.to_vector(), pb = m_args[i].pb.to_vector();
            b200::check(ltg_dotprod(m_args[i].a->handle(), pa.data(), m_args[i].b->handle(), pb.data(), &v[i]));
        }
    }
    double calculate() {
        std::vector<double> v;
        calculate(v);
        return v.at(0);
    }
};


// ---------------------------------------------------------------- letter interface
//
// The expression layer libtensor users write (libtensor/expr/iface/letter.h,
// label.h; libtensor/expr/operators/contract.h, dot_product.h, plus_minus.h,
// multiply_divide.h):
//     letter i, j, a, b, c, d;
//     r(i|j|a|b) = 0.5 * contract(c|d, t(i|j|c|d), v(a|b|c|d));
//     r(i|j|a|b) += x(i|j|a|b) - x(j|i|a|b);
//     double e = dot_product(t(i|j|a|b), r(i|j|a|b));
// An assignment evaluates its terms directly with the operations above: each
// contraction term with one btod_contract2 (the first term assigns, the rest
// add), all tensor terms together with one btod_add.  Contraction operands
// are (scaled) tensors; the result must not appear on the right-hand side.

// Letters are told apart by identity (address).
class letter {
public:
    letter() { }
    letter(const letter &) = delete;
    letter &operator=(const letter &) = delete;
};

template<size_t N>
class label {
    std::array<const letter *, N> m_l;
public:
    label() { m_l.fill(nullptr); }
    explicit label(const letter &l) { static_assert(N == 1, "one letter"); m_l[0] = &l; }
    const letter &letter_at(size_t i) const { return *m_l.at(i); }
    const letter *ptr(size_t i) const { return m_l[i]; }
    void set(size_t i, const letter *l) { m_l.at(i) = l; }
    bool contains(const letter &l) const {
        for (size_t i = 0; i < N; i++) if (m_l[i] == &l) return true;
        return false;
    }
    size_t index_of(const letter &l) const {
        for (size_t i = 0; i < N; i++) if (m_l[i] == &l) return i;
        throw bad_parameter("label: letter not found");
    }
    template<size_t M> friend class label;
    template<size_t M> label<M + 1> append(const letter &l) const;
    friend inline label<2> operator|(const letter &l1, const letter &l2);
    template<size_t M> friend label<M + 1> operator|(const label<M> &e, const letter &l);
};

inline label<2> operator|(const letter &l1, const letter &l2) {
    if (&l1 == &l2) throw bad_parameter("operator|: repeated letter");
    label<2> r;
    r.m_l[0] = &l1;
    r.m_l[1] = &l2;
    return r;
}

template<size_t N>
label<N + 1> operator|(const label<N> &e, const letter &l) {
    if (e.contains(l)) throw bad_parameter("operator|: repeated letter");
    label<N + 1> r;
    for (size_t i = 0; i < N; i++) r.m_l[i] = e.m_l[i];
    r.m_l[N] = &l;
    return r;
}

// btensor<N> is the block tensor of double
template<size_t N, typename T = double>
using btensor = block_tensor<N, T>;

namespace b200 {

// CUDA graph of a sequence of operations (ltg_graph_begin/end/launch): run
// every operation once before the capture (their plans are built then), capture
// the sequence, then launch it as often as needed.
class graph {
    ltg_graph *m_g = nullptr;
public:
    explicit graph(ltg_graph *g) : m_g(g) { }
    graph(graph &&o) noexcept : m_g(o.m_g) { o.m_g = nullptr; }
    graph(const graph &) = delete;
    graph &operator=(const graph &) = delete;
    ~graph() { if (m_g) ltg_graph_destroy(m_g); }
    void launch() { check(ltg_graph_launch(m_g)); }
};
inline void begin_capture() { check(ltg_graph_begin(context())); }
inline graph end_capture() {
    ltg_graph *g = nullptr;
    check(ltg_graph_end(context(), &g));
    return graph(g);
}
inline void synchronize() { check(ltg_ctx_synchronize(context())); }

// Arithmetic of the letter interface's contractions (ltg.h modes; default
// LTG_MODE_PLAIN_FP64, the FP64 drop-in path).
struct expr_precision { int32_t mode = LTG_MODE_PLAIN_FP64, nslices = 0; };
inline expr_precision &letter_precision() { static expr_precision p; return p; }
inline void set_letter_precision(int32_t mode, int32_t nslices) {
    letter_precision().mode = mode;
    letter_precision().nslices = nslices;
}
}  // namespace b200

namespace expr_detail {

// Permutation taking a tensor labelled `from` to the order of `to`:
// result index d comes from source index perm[d].
template<size_t N>
permutation<N> align(const label<N> &from, const label<N> &to) {
    std::vector<size_t> v(N);
    for (size_t d = 0; d < N; d++) v[d] = from.index_of(to.letter_at(d));
    return permutation<N>(v);
}

// Letter pairs exchanged by a (anti)symmetrizer.
struct letter_swap {
    std::vector<std::pair<const letter *, const letter *> > pairs;
    const letter *map(const letter *l) const {
        for (const auto &p : pairs) {
            if (l == p.first) return p.second;
            if (l == p.second) return p.first;
        }
        return l;
    }
};

template<size_t N>
label<N> relabel(const label<N> &l, const letter_swap &sw) {
    label<N> r = l;
    for (size_t i = 0; i < N; i++) r.set(i, sw.map(l.ptr(i)));
    return r;
}

// One dimension of a block index space: its extent and split points.
struct dim_space {
    size_t dim = 0;
    std::vector<size_t> splits;
};
template<size_t N>
dim_space dim_of(const block_index_space<N> &b, size_t i) {
    dim_space d;
    d.dim = b.get_dims()[i];
    d.splits = b.get_splits(i);
    return d;
}
template<size_t N>
block_index_space<N> make_space(const std::vector<dim_space> &d) {
    index<N> i1;
    for (size_t i = 0; i < N; i++) i1[i] = d[i].dim - 1;
    block_index_space<N> bis(dimensions<N>(index_range<N>(index<N>(), i1)));
    for (size_t i = 0; i < N; i++) {
        mask<N> m;
        m[i] = true;
        for (size_t x : d[i].splits) bis.split(m, x);
    }
    return bis;
}

// The operations of one assignment in order, each run as it is added (later
// operations use the tensors earlier ones created), with the operation
// objects and intermediates kept, so that the sequence can run again and be
// captured as one CUDA graph (b200::assignment).
struct program {
    std::vector<std::function<void()> > steps;
    std::vector<std::shared_ptr<void> > keep;
    void add(std::function<void()> f) {
        f();
        steps.push_back(std::move(f));
    }
    void run() const {
        for (const auto &f : steps) f();
    }
};

template<size_t N> struct tensor_term;

// One term of an expression of order N.
template<size_t N>
struct term {
    double coeff = 1.0;
    virtual ~term() { }
    virtual bool uses(const void *bt) const = 0;
    virtual term *scaled(double f) const = 0;
    // the term with the letters of sw exchanged (the permuted term P E)
    virtual term *swapped(const letter_swap &sw) const = 0;
    // its letters in their natural order (an operand's own order; a
    // contraction's: A's free letters, then B's)
    virtual label<N> natural_label() const = 0;
    // contraction terms: the operations that write the term into c (assign,
    // or add d times the term), appended to pg
    virtual bool is_contraction() const = 0;
    virtual void contract_into(program &pg, block_tensor<N, double> &c, const label<N> &lc, bool add,
                               double d) const = 0;
    // contraction terms: the term as an intermediate labelled l
    virtual tensor_term<N> contract_temp(program &pg, const label<N> &l) const = 0;
};

template<size_t N>
struct tensor_term : term<N> {
    block_tensor<N, double> *bt;
    label<N> lab;
    tensor_term(block_tensor<N, double> &t, const label<N> &l) : bt(&t), lab(l) { }
    bool uses(const void *p) const override { return p == (const void *)bt; }
    term<N> *scaled(double f) const override {
        tensor_term *r = new tensor_term(*this);
        r->coeff *= f;
        return r;
    }
    term<N> *swapped(const letter_swap &sw) const override {
        tensor_term *r = new tensor_term(*this);
        r->lab = relabel(lab, sw);
        return r;
    }
    label<N> natural_label() const override { return lab; }
    bool is_contraction() const override { return false; }
    void contract_into(program &, block_tensor<N, double> &, const label<N> &, bool, double) const override {
        throw exception("tensor term evaluated as a contraction");
    }
    tensor_term<N> contract_temp(program &, const label<N> &) const override {
        throw exception("tensor term evaluated as a contraction");
    }
};

}  // namespace expr_detail

// Right-hand side of order N: a sum of (scaled) tensor, contraction and
// symmetrizer terms.
template<size_t N, typename T = double>
class expr_rhs {
    static_assert(sizeof(T) == 8, "expressions of double");
public:
    std::vector<std::shared_ptr<expr_detail::term<N> > > terms;
    expr_rhs() { }
    explicit expr_rhs(expr_detail::term<N> *t) { terms.emplace_back(t); }
    // the single tensor of a (scaled) tensor expression
    const expr_detail::tensor_term<N> &as_tensor(const char *what) const {
        const expr_detail::tensor_term<N> *t =
            terms.size() == 1 ? dynamic_cast<const expr_detail::tensor_term<N> *>(terms[0].get()) : nullptr;
        if (!t) throw bad_parameter(std::string(what) + ": operands must be (scaled) tensors");
        return *t;
    }
    bool uses(const void *p) const {
        for (const auto &t : terms) if (t->uses(p)) return true;
        return false;
    }
    // the letters of the expression: those of its first term, which every
    // other term must have too (in any order)
    label<N> natural_label() const {
        if (terms.empty()) throw bad_parameter("empty expression");
        const label<N> l = terms[0]->natural_label();
        for (const auto &t : terms) {
            const label<N> m = t->natural_label();
            for (size_t i = 0; i < N; i++)
                if (!l.contains(m.letter_at(i))) throw bad_parameter("terms of a sum with different letters");
        }
        return l;
    }
};

namespace expr_detail {

// E + sign P E for the letter exchange P: holds E (evaluated with the
// target's letters; contraction terms of E once, into a temporary)
template<size_t N>
struct symm_term : term<N> {
    expr_rhs<N> sub;
    letter_swap sw;
    double sign;
    symm_term(const expr_rhs<N> &e, const letter_swap &s, double sg) : sub(e), sw(s), sign(sg) { }
    bool uses(const void *p) const override { return sub.uses(p); }
    term<N> *scaled(double f) const override {
        symm_term *r = new symm_term(*this);
        r->coeff *= f;
        return r;
    }
    term<N> *swapped(const letter_swap &s2) const override {
        expr_rhs<N> e;
        for (const auto &t : sub.terms) e.terms.emplace_back(t->swapped(s2));
        letter_swap s = sw;
        for (auto &p : s.pairs) p = std::make_pair(s2.map(p.first), s2.map(p.second));
        symm_term *r = new symm_term(e, s, sign);
        r->coeff = this->coeff;
        return r;
    }
    label<N> natural_label() const override { return sub.natural_label(); }
    bool is_contraction() const override { return false; }
    void contract_into(program &, block_tensor<N, double> &, const label<N> &, bool, double) const override {
        throw exception("symmetrizer evaluated as a contraction");
    }
    tensor_term<N> contract_temp(program &, const label<N> &) const override {
        throw exception("symmetrizer evaluated as a contraction");
    }
};

// The terms of e (times f) as contraction terms and (scaled) tensor terms;
// symmetrizers are expanded, the contraction terms inside them evaluated once
// into intermediates labelled l.
template<size_t N>
void flatten(const expr_rhs<N> &e, double f, const label<N> &l, program &pg,
             std::vector<std::shared_ptr<term<N> > > &contr, std::vector<tensor_term<N> > &tens) {
    for (const auto &t : e.terms) {
        if (t->is_contraction()) { contr.emplace_back(t->scaled(f)); continue; }
        if (const tensor_term<N> *x = dynamic_cast<const tensor_term<N> *>(t.get())) {
            tens.push_back(*x);
            tens.back().coeff *= f;
            continue;
        }
        const symm_term<N> &y = dynamic_cast<const symm_term<N> &>(*t);
        std::vector<std::shared_ptr<term<N> > > sc;
        std::vector<tensor_term<N> > st;
        flatten(y.sub, 1.0, l, pg, sc, st);
        for (const auto &c : sc) st.push_back(c->contract_temp(pg, l));
        for (const tensor_term<N> &x : st) {
            tens.push_back(x);
            tens.back().coeff *= f * y.coeff;
            tens.push_back(x);
            tens.back().lab = relabel(x.lab, y.sw);
            tens.back().coeff *= f * y.coeff * y.sign;
        }
    }
}

// An intermediate holding the sum of tensor terms, labelled l: the block
// index space of the terms and the symmetry common to all of them
// (ltg_bt_create_sum_space), assigned with one btod_add.
template<size_t N>
tensor_term<N> sum_temp(program &pg, const std::vector<tensor_term<N> > &tens, const label<N> &l) {
    std::vector<ltg_bt *> hs;
    std::vector<int32_t> perms;
    for (const tensor_term<N> &x : tens) {
        hs.push_back(x.bt->handle());
        const std::vector<int32_t> p = align(x.lab, l).to_vector();
        perms.insert(perms.end(), p.begin(), p.end());
    }
    const permutation<N> p0 = align(tens[0].lab, l);
    std::vector<dim_space> d(N);
    for (size_t i = 0; i < N; i++) d[i] = dim_of(tens[0].bt->get_bis(), p0.to_vector()[i]);
    std::shared_ptr<block_tensor<N, double> > tmp(new block_tensor<N, double>(make_space<N>(d)));
    ltg_bt *h = nullptr;
    b200::check(ltg_bt_create_sum_space((int32_t)hs.size(), hs.data(), perms.data(), &h));
    tmp->adopt(h);
    std::shared_ptr<btod_add<N> > op;
    for (const tensor_term<N> &x : tens) {
        if (!op) op.reset(new btod_add<N>(*x.bt, align(x.lab, l), x.coeff));
        else op->add_op(*x.bt, align(x.lab, l), x.coeff);
    }
    pg.keep.push_back(tmp);
    pg.keep.push_back(op);
    block_tensor<N, double> *t = tmp.get();
    btod_add<N> *o = op.get();
    pg.add([o, t] { o->perform(*t); });
    return tensor_term<N>(*t, l);
}

// The expression as one (scaled) tensor: itself when it is one, else an
// intermediate labelled with its natural letters.
template<size_t N>
tensor_term<N> materialize(const expr_rhs<N> &e, program &pg) {
    if (e.terms.size() == 1)
        if (const tensor_term<N> *x = dynamic_cast<const tensor_term<N> *>(e.terms[0].get())) return *x;
    const label<N> l = e.natural_label();
    std::vector<std::shared_ptr<term<N> > > contr;
    std::vector<tensor_term<N> > tens;
    flatten(e, 1.0, l, pg, contr, tens);
    for (const auto &c : contr) tens.push_back(c->contract_temp(pg, l));
    if (tens.size() == 1) return tens[0];
    return sum_temp(pg, tens, l);
}

}  // namespace expr_detail

template<size_t N>
class labeled_btensor {
    block_tensor<N, double> &m_bt;
    label<N> m_label;
public:
    // The operations of  this = e  (add: this += sign e) appended to pg.
    void evaluate(expr_detail::program &pg, const expr_rhs<N> &e, bool add, double sign) {
        if (e.uses(&m_bt)) {
            // the result on the right-hand side: the whole expression into an
            // intermediate first, then into the result
            const expr_detail::tensor_term<N> x = expr_detail::materialize(e, pg);
            std::shared_ptr<btod_add<N> > op(new btod_add<N>(*x.bt, expr_detail::align(x.lab, m_label), x.coeff));
            pg.keep.push_back(op);
            btod_add<N> *o = op.get();
            block_tensor<N, double> *r = &m_bt;
            if (add) pg.add([o, r, sign] { o->perform(*r, sign); });
            else if (sign == 1.0) pg.add([o, r] { o->perform(*r); });
            else pg.add([o, r, sign] { b200::check(ltg_bt_set_zero(r->handle())); o->perform(*r, sign); });
            return;
        }
        std::vector<std::shared_ptr<expr_detail::term<N> > > contr;
        std::vector<expr_detail::tensor_term<N> > tens;
        expr_detail::flatten(e, 1.0, m_label, pg, contr, tens);
        bool written = add;
        for (const auto &t : contr) {
            t->contract_into(pg, m_bt, m_label, written, sign);
            written = true;
        }
        std::shared_ptr<btod_add<N> > sum;
        for (const expr_detail::tensor_term<N> &x : tens) {
            const permutation<N> p = expr_detail::align(x.lab, m_label);
            if (!sum) sum.reset(new btod_add<N>(*x.bt, p, x.coeff));
            else sum->add_op(*x.bt, p, x.coeff);
        }
        block_tensor<N, double> *r = &m_bt;
        if (!sum) {
            if (!written) pg.add([r] { b200::check(ltg_bt_set_zero(r->handle())); });
            return;
        }
        pg.keep.push_back(sum);
        btod_add<N> *o = sum.get();
        if (written) pg.add([o, r, sign] { o->perform(*r, sign); });
        else if (sign == 1.0) pg.add([o, r] { o->perform(*r); });
        else pg.add([o, r, sign] {
            // assignment of a negated sum: C = 0 - ... is C += -sum after zeroing
            b200::check(ltg_bt_set_zero(r->handle()));
            o->perform(*r, sign);
        });
    }
    labeled_btensor(block_tensor<N, double> &bt, const label<N> &l) : m_bt(bt), m_label(l) { }
    block_tensor<N, double> &get_btensor() const { return m_bt; }
    const label<N> &get_label() const { return m_label; }
    operator expr_rhs<N>() const { return expr_rhs<N>(new expr_detail::tensor_term<N>(m_bt, m_label)); }
    labeled_btensor &operator=(const expr_rhs<N> &e) { expr_detail::program pg; evaluate(pg, e, false, 1.0); return *this; }
    labeled_btensor &operator=(const labeled_btensor &o) { return *this = expr_rhs<N>(o); }
    labeled_btensor &operator+=(const expr_rhs<N> &e) { expr_detail::program pg; evaluate(pg, e, true, 1.0); return *this; }
    labeled_btensor &operator-=(const expr_rhs<N> &e) { expr_detail::program pg; evaluate(pg, e, true, -1.0); return *this; }
};

template<size_t N, typename T>
template<size_t M>
labeled_btensor<M> block_tensor<N, T>::operator()(const label<M> &l) {
    static_assert(M == N, "a label needs one letter per tensor index");
    return labeled_btensor<M>(*this, l);
}

// sums and scalar multiples
template<size_t N>
expr_rhs<N> operator+(const expr_rhs<N> &a, const expr_rhs<N> &b) {
    expr_rhs<N> r(a);
    r.terms.insert(r.terms.end(), b.terms.begin(), b.terms.end());
    return r;
}
template<size_t N>
expr_rhs<N> operator*(double f, const expr_rhs<N> &a) {
    expr_rhs<N> r;
    for (const auto &t : a.terms) r.terms.emplace_back(t->scaled(f));
    return r;
}
template<size_t N> expr_rhs<N> operator*(const expr_rhs<N> &a, double f) { return f * a; }
template<size_t N> expr_rhs<N> operator-(const expr_rhs<N> &a) { return -1.0 * a; }
template<size_t N> expr_rhs<N> operator-(const expr_rhs<N> &a, const expr_rhs<N> &b) { return a + (-1.0 * b); }
template<size_t N> expr_rhs<N> operator+(const labeled_btensor<N> &a, const labeled_btensor<N> &b) { return expr_rhs<N>(a) + expr_rhs<N>(b); }
template<size_t N> expr_rhs<N> operator-(const labeled_btensor<N> &a, const labeled_btensor<N> &b) { return expr_rhs<N>(a) - expr_rhs<N>(b); }
template<size_t N> expr_rhs<N> operator+(const expr_rhs<N> &a, const labeled_btensor<N> &b) { return a + expr_rhs<N>(b); }
template<size_t N> expr_rhs<N> operator-(const expr_rhs<N> &a, const labeled_btensor<N> &b) { return a - expr_rhs<N>(b); }
template<size_t N> expr_rhs<N> operator+(const labeled_btensor<N> &a, const expr_rhs<N> &b) { return expr_rhs<N>(a) + b; }
template<size_t N> expr_rhs<N> operator-(const labeled_btensor<N> &a, const expr_rhs<N> &b) { return expr_rhs<N>(a) - b; }
template<size_t N> expr_rhs<N> operator*(double f, const labeled_btensor<N> &a) { return f * expr_rhs<N>(a); }
template<size_t N> expr_rhs<N> operator*(const labeled_btensor<N> &a, double f) { return f * expr_rhs<N>(a); }
template<size_t N> expr_rhs<N> operator-(const labeled_btensor<N> &a) { return -1.0 * expr_rhs<N>(a); }

namespace b200 {

// One letter-interface assignment kept for repeated runs: constructing it
// evaluates  lhs = rhs  (mode 0; +1: +=, -1: -=) once, keeping every
// operation and intermediate (nested contractions, contractions of sums,
// symmetrizers); run() evaluates it again with the same operations, and
// after capture() run() launches the whole assignment as one CUDA graph.
// The tensors named in the expression must outlive the object.
template<size_t N>
class assignment {
    std::shared_ptr<expr_detail::program> m_pg;
    std::unique_ptr<graph> m_graph;
public:
    assignment(labeled_btensor<N> lhs, const expr_rhs<N> &rhs, int mode = 0) : m_pg(new expr_detail::program()) {
        lhs.evaluate(*m_pg, rhs, mode != 0, mode < 0 ? -1.0 : 1.0);
    }
    void run() {
        if (m_graph) m_graph->launch();
        else m_pg->run();
    }
    void capture() {
        begin_capture();
        try {
            m_pg->run();
        } catch (...) {
            end_capture();
            throw;
        }
        m_graph.reset(new graph(end_capture()));
    }
    size_t operations() const { return m_pg->steps.size(); }
};
}  // namespace b200

namespace expr_detail {

// contraction of A (order NA) and B (order NB) over K letters; A and B are
// expressions (intermediates evaluated first when they are not tensors)
template<size_t NA, size_t NB, size_t K>
struct contract_term : term<NA + NB - 2 * K> {
    static constexpr size_t NC = NA + NB - 2 * K;
    expr_rhs<NA> ea;
    expr_rhs<NB> eb;
    label<NA> la;
    label<NB> lb;
    label<K> lk;
    contract_term(const expr_rhs<NA> &x, const expr_rhs<NB> &y, const label<K> &k)
        : ea(x), eb(y), la(x.natural_label()), lb(y.natural_label()), lk(k) {
        for (size_t i = 0; i < K; i++)
            if (!la.contains(lk.letter_at(i)) || !lb.contains(lk.letter_at(i)))
                throw bad_parameter("contract: a contracted letter is missing from an operand");
    }
    bool uses(const void *p) const override { return ea.uses(p) || eb.uses(p); }
    term<NC> *scaled(double f) const override {
        contract_term *r = new contract_term(*this);
        r->coeff *= f;
        return r;
    }
    term<NC> *swapped(const letter_swap &sw) const override {
        for (size_t i = 0; i < K; i++)
            if (sw.map(lk.ptr(i)) != lk.ptr(i)) throw bad_parameter("symm/asymm: a contracted letter is exchanged");
        expr_rhs<NA> xa;
        expr_rhs<NB> xb;
        for (const auto &t : ea.terms) xa.terms.emplace_back(t->swapped(sw));
        for (const auto &t : eb.terms) xb.terms.emplace_back(t->swapped(sw));
        contract_term *r = new contract_term(xa, xb, lk);
        r->coeff = this->coeff;
        return r;
    }
    label<NC> natural_label() const override {
        label<NC> l;
        size_t k = 0;
        for (size_t i = 0; i < NA; i++) if (!lk.contains(la.letter_at(i))) l.set(k++, la.ptr(i));
        for (size_t i = 0; i < NB; i++) if (!lk.contains(lb.letter_at(i))) l.set(k++, lb.ptr(i));
        if (k != NC) throw bad_parameter("contract: uncontracted letters do not match the result");
        return l;
    }
    bool is_contraction() const override { return true; }
    void contract_into(program &pg, block_tensor<NC, double> &c, const label<NC> &lc, bool add,
                       double d) const override {
        const tensor_term<NA> x = materialize(ea, pg);
        const tensor_term<NB> y = materialize(eb, pg);
        // natural result order: A's free letters, then B's (contraction2)
        std::vector<const letter *> nat;
        for (size_t i = 0; i < NA; i++) if (!lk.contains(x.lab.letter_at(i))) nat.push_back(x.lab.ptr(i));
        for (size_t i = 0; i < NB; i++) if (!lk.contains(y.lab.letter_at(i))) nat.push_back(y.lab.ptr(i));
        if (nat.size() != NC) throw bad_parameter("contract: uncontracted letters do not match the result");
        std::vector<size_t> pc(NC);
        for (size_t dd = 0; dd < NC; dd++) {
            size_t k = NC;
            for (size_t q = 0; q < NC; q++) if (nat[q] == lc.ptr(dd)) k = q;
            if (k == NC) throw bad_parameter("contract: result letter not produced by the contraction");
            pc[dd] = k;
        }
        contraction2<NA - K, NB - K, K> contr{permutation<NC>(pc)};
        for (size_t i = 0; i < K; i++) contr.contract(x.lab.index_of(lk.letter_at(i)), y.lab.index_of(lk.letter_at(i)));
        std::shared_ptr<btod_contract2<NA - K, NB - K, K> > op(
            new btod_contract2<NA - K, NB - K, K>(contr, *x.bt, 1.0, *y.bt, 1.0, this->coeff * x.coeff * y.coeff));
        op->set_split_precision(b200::letter_precision().mode, b200::letter_precision().nslices);
        pg.keep.push_back(op);
        btod_contract2<NA - K, NB - K, K> *o = op.get();
        block_tensor<NC, double> *t = &c;
        if (add) pg.add([o, t, d] { o->perform(*t, d); });
        else if (d == 1.0) pg.add([o, t] { o->perform(*t); });
        else pg.add([o, t, d] {
            o->perform(*t);
            b200::check(ltg_scale(t->handle(), d));
        });
    }
    tensor_term<NC> contract_temp(program &pg, const label<NC> &l) const override {
        // the intermediate's index space from the operands' dims (their
        // letters' dims); its symmetry is the contraction's result symmetry,
        // taken on by the assignment
        const tensor_term<NA> x = materialize(ea, pg);
        const tensor_term<NB> y = materialize(eb, pg);
        std::vector<dim_space> d(NC);
        for (size_t i = 0; i < NC; i++) {
            const letter &w = l.letter_at(i);
            if (x.lab.contains(w)) d[i] = dim_of(x.bt->get_bis(), x.lab.index_of(w));
            else d[i] = dim_of(y.bt->get_bis(), y.lab.index_of(w));
        }
        std::shared_ptr<block_tensor<NC, double> > tmp(new block_tensor<NC, double>(make_space<NC>(d)));
        pg.keep.push_back(tmp);
        expr_rhs<NA> xa;
        xa.terms.emplace_back(new tensor_term<NA>(x));
        expr_rhs<NB> xb;
        xb.terms.emplace_back(new tensor_term<NB>(y));
        contract_term done(xa, xb, lk);
        done.coeff = this->coeff;
        done.contract_into(pg, *tmp, l, false, 1.0);
        return tensor_term<NC>(*tmp, l);
    }
};

}  // namespace expr_detail

// contract(letters, A(...), B(...)) (libtensor/expr/operators/contract.h);
// A and B may be any expressions (sums, contractions, symmetrizers), which
// are evaluated into intermediates first
template<size_t K, size_t NA, size_t NB>
expr_rhs<NA + NB - 2 * K> contract(const label<K> &lk, const expr_rhs<NA> &a, const expr_rhs<NB> &b) {
    static_assert(K >= 1 && K <= NA && K <= NB && NA + NB > 2 * K, "contraction orders");
    return expr_rhs<NA + NB - 2 * K>(new expr_detail::contract_term<NA, NB, K>(a, b, lk));
}
template<size_t NA, size_t NB>
expr_rhs<NA + NB - 2> contract(const letter &l, const expr_rhs<NA> &a, const expr_rhs<NB> &b) {
    return contract(label<1>(l), a, b);
}
template<size_t K, size_t NA, size_t NB>
expr_rhs<NA + NB - 2 * K> contract(const label<K> &lk, const labeled_btensor<NA> &a, const labeled_btensor<NB> &b) {
    return contract(lk, expr_rhs<NA>(a), expr_rhs<NB>(b));
}
template<size_t K, size_t NA, size_t NB>
expr_rhs<NA + NB - 2 * K> contract(const label<K> &lk, const expr_rhs<NA> &a, const labeled_btensor<NB> &b) {
    return contract(lk, a, expr_rhs<NB>(b));
}
template<size_t K, size_t NA, size_t NB>
expr_rhs<NA + NB - 2 * K> contract(const label<K> &lk, const labeled_btensor<NA> &a, const expr_rhs<NB> &b) {
    return contract(lk, expr_rhs<NA>(a), b);
}
template<size_t NA, size_t NB>
expr_rhs<NA + NB - 2> contract(const letter &l, const labeled_btensor<NA> &a, const labeled_btensor<NB> &b) {
    return contract(label<1>(l), expr_rhs<NA>(a), expr_rhs<NB>(b));
}
template<size_t NA, size_t NB>
expr_rhs<NA + NB - 2> contract(const letter &l, const expr_rhs<NA> &a, const labeled_btensor<NB> &b) {
    return contract(label<1>(l), a, expr_rhs<NB>(b));
}
template<size_t NA, size_t NB>
expr_rhs<NA + NB - 2> contract(const letter &l, const labeled_btensor<NA> &a, const expr_rhs<NB> &b) {
    return contract(label<1>(l), expr_rhs<NA>(a), b);
}

// dot_product(A(...), B(...)) (libtensor/expr/operators/dot_product.h);
// operands that are not tensors are evaluated into intermediates first
template<size_t N>
double dot_product(const expr_rhs<N> &a, const expr_rhs<N> &b) {
    expr_detail::program pg;
    const expr_detail::tensor_term<N> x = expr_detail::materialize(a, pg);
    const expr_detail::tensor_term<N> y = expr_detail::materialize(b, pg);
    return x.coeff * y.coeff *
           btod_dotprod<N>(*x.bt, permutation<N>(), *y.bt, expr_detail::align(y.lab, x.lab)).calculate();
}
template<size_t N>
double dot_product(const labeled_btensor<N> &a, const labeled_btensor<N> &b) {
    return dot_product(expr_rhs<N>(a), expr_rhs<N>(b));
}
template<size_t N>
double dot_product(const expr_rhs<N> &a, const labeled_btensor<N> &b) { return dot_product(a, expr_rhs<N>(b)); }
template<size_t N>
double dot_product(const labeled_btensor<N> &a, const expr_rhs<N> &b) { return dot_product(expr_rhs<N>(a), b); }

// symm / asymm (libtensor/expr/operators/symm_asymm.h): E + P E and E - P E,
// P exchanging the letters of l1 with those of l2 (pairwise, simultaneously)
template<size_t N, size_t M>
expr_rhs<N> symm(const label<M> &l1, const label<M> &l2, const expr_rhs<N> &e) {
    expr_detail::letter_swap sw;
    for (size_t i = 0; i < M; i++) sw.pairs.push_back(std::make_pair(l1.ptr(i), l2.ptr(i)));
    return expr_rhs<N>(new expr_detail::symm_term<N>(e, sw, 1.0));
}
template<size_t N, size_t M>
expr_rhs<N> asymm(const label<M> &l1, const label<M> &l2, const expr_rhs<N> &e) {
    expr_detail::letter_swap sw;
    for (size_t i = 0; i < M; i++) sw.pairs.push_back(std::make_pair(l1.ptr(i), l2.ptr(i)));
    return expr_rhs<N>(new expr_detail::symm_term<N>(e, sw, -1.0));
}
template<size_t N>
expr_rhs<N> symm(const letter &l1, const letter &l2, const expr_rhs<N> &e) { return symm(label<1>(l1), label<1>(l2), e); }
template<size_t N>
expr_rhs<N> asymm(const letter &l1, const letter &l2, const expr_rhs<N> &e) { return asymm(label<1>(l1), label<1>(l2), e); }
template<size_t N, size_t M>
expr_rhs<N> symm(const label<M> &l1, const label<M> &l2, const labeled_btensor<N> &e) { return symm(l1, l2, expr_rhs<N>(e)); }
template<size_t N, size_t M>
expr_rhs<N> asymm(const label<M> &l1, const label<M> &l2, const labeled_btensor<N> &e) { return asymm(l1, l2, expr_rhs<N>(e)); }
template<size_t N>
expr_rhs<N> symm(const letter &l1, const letter &l2, const labeled_btensor<N> &e) { return symm(l1, l2, expr_rhs<N>(e)); }
template<size_t N>
expr_rhs<N> asymm(const letter &l1, const letter &l2, const labeled_btensor<N> &e) { return asymm(l1, l2, expr_rhs<N>(e)); }

namespace b200 {

// Symmetrizer of a tensor or of an operation's result (ltg_symmetrize): the
// group of the exchange of two indexes, of a unitary permutation, or of the
// 24 permutations of four indexes.  An operation is evaluated into a result
// tensor the object keeps (its own result space), then summed over the
// group; assigning gives B the symmetrized space (as the reference's
// perform does), repeated assignments reuse it.
template<size_t N>
class symmetrizer : public additive_bto<N> {
    block_tensor<N, double> *m_a = nullptr;          // a tensor, or
    additive_bto<N> *m_op = nullptr;                 // an operation evaluated into m_tmp
    std::unique_ptr<block_tensor<N, double> > m_tmp;
    int32_t m_nidx;
    std::vector<int32_t> m_idx;
    bool m_symm;
    ltg_bt *m_adopted = nullptr;
    block_tensor<N, double> &source(block_tensor<N, double> &btb) {
        if (m_a) return *m_a;
        if (!m_tmp) m_tmp.reset(new block_tensor<N, double>(btb.get_bis()));
        m_op->perform(*m_tmp);
        return *m_tmp;
    }
protected:
    symmetrizer(block_tensor<N, double> *a, additive_bto<N> *op, int32_t nidx, std::vector<int32_t> idx, bool symm)
        : m_a(a), m_op(op), m_nidx(nidx), m_idx(std::move(idx)), m_symm(symm) { }
public:
    void perform(block_tensor<N, double> &btb) override {
        // an operation that forms the symmetrized sum itself (a contraction
        // writing both terms from its epilogue) needs no temporary
        if (m_op && m_op->perform_symmetrized(btb, m_nidx, m_idx.data(), m_symm, &m_adopted)) return;
        block_tensor<N, double> &a = source(btb);
        if (!(btb.is_bound() && btb.handle() == m_adopted)) {
            ltg_bt *b = nullptr;
            check(ltg_bt_create_symmetrized(a.handle(), m_nidx, m_idx.data(), m_symm ? 1 : 0, &b));
            btb.adopt(b);
            m_adopted = b;
        }
        check(ltg_symmetrize(a.handle(), 1.0, m_nidx, m_idx.data(), m_symm ? 1 : 0, btb.handle(), 0, 0.0));
    }
    void perform(block_tensor<N, double> &btb, double d) override {
        block_tensor<N, double> &a = source(btb);
        check(ltg_symmetrize(a.handle(), 1.0, m_nidx, m_idx.data(), m_symm ? 1 : 0, btb.handle(), 1, d));
    }
};

inline std::vector<int32_t> idx_vec(std::initializer_list<size_t> l) {
    std::vector<int32_t> v;
    for (size_t x : l) v.push_back((int32_t)x);
    return v;
}
template<size_t N>
std::vector<int32_t> perm_vec(const permutation<N> &p) { return p.to_vector(); }
}  // namespace b200

// btod_symmetrize2 (libtensor/block_tensor/btod_symmetrize2.h:19-60):
// B = A + P(A) (symm) or A - P(A) for the exchange of indexes i1 and i2 or a
// unitary permutation P, A an operation's result or a tensor.
template<size_t N>
class btod_symmetrize2 : public b200::symmetrizer<N> {
public:
    btod_symmetrize2(additive_bto<N> &op, size_t i1, size_t i2, bool symm)
        : b200::symmetrizer<N>(nullptr, &op, 2, b200::idx_vec({i1, i2}), symm) { }
    btod_symmetrize2(additive_bto<N> &op, const permutation<N> &perm, bool symm)
        : b200::symmetrizer<N>(nullptr, &op, -1, b200::perm_vec(perm), symm) { }
    btod_symmetrize2(block_tensor<N, double> &bta, size_t i1, size_t i2, bool symm)
        : b200::symmetrizer<N>(&bta, nullptr, 2, b200::idx_vec({i1, i2}), symm) { }
    btod_symmetrize2(block_tensor<N, double> &bta, const permutation<N> &perm, bool symm)
        : b200::symmetrizer<N>(&bta, nullptr, -1, b200::perm_vec(perm), symm) { }
};

// btod_symmetrize4 (libtensor/block_tensor/btod_symmetrize4.h:27-60): the sum
// over the 24 permutations of indexes i1..i4 (with the permutation's parity
// as sign when not symm) of A, an operation's result or a tensor.
template<size_t N>
class btod_symmetrize4 : public b200::symmetrizer<N> {
public:
    btod_symmetrize4(additive_bto<N> &op, size_t i1, size_t i2, size_t i3, size_t i4, bool symm)
        : b200::symmetrizer<N>(nullptr, &op, 4, b200::idx_vec({i1, i2, i3, i4}), symm) { }
    btod_symmetrize4(block_tensor<N, double> &bta, size_t i1, size_t i2, size_t i3, size_t i4, bool symm)
        : b200::symmetrizer<N>(&bta, nullptr, 4, b200::idx_vec({i1, i2, i3, i4}), symm) { }
};

// Result block index space of a contraction: A's uncontracted dims, then
// B's, permuted by the contraction's permc.
template<size_t N, size_t M, size_t K>
block_index_space<N + M> contraction_space(const contraction2<N, M, K> &contr,
                                           const block_index_space<N + K> &bisa,
                                           const block_index_space<M + K> &bisb) {
    std::vector<bool> ca(N + K, false), cb(M + K, false);
    for (const std::pair<size_t, size_t> &p : contr.get_pairs()) {
        ca[p.first] = true;
        cb[p.second] = true;
    }
    std::vector<expr_detail::dim_space> nat;
    for (size_t i = 0; i < N + K; i++) if (!ca[i]) nat.push_back(expr_detail::dim_of(bisa, i));
    for (size_t i = 0; i < M + K; i++) if (!cb[i]) nat.push_back(expr_detail::dim_of(bisb, i));
    const std::vector<int32_t> pc = contr.get_permc().to_vector();
    std::vector<expr_detail::dim_space> d(N + M);
    for (size_t i = 0; i < N + M; i++) d[i] = nat[(size_t)pc[i]];
    return expr_detail::make_space<N + M>(d);
}

// btod_contract3 (libtensor/block_tensor/btod_contract3.h:36): D = kd (AB) C
// with AB = contr1(A, B) and D = contr2(AB, C).  The intermediate AB is one
// device tensor the operation keeps (it is formed whole: the reference forms
// it in batches of B's blocks to bound host memory, which 180 GB of HBM
// makes unnecessary at these sizes); the second contraction is built on the
// first perform, when AB's non-zero blocks are known, and reused.
template<size_t N1, size_t N2, size_t N3, size_t K1, size_t K2>
class btod_contract3 : public additive_bto<N1 + N2 + N3> {
    static constexpr size_t NAB = N1 + N2 + K2;
    contraction2<N1 + N2, N3, K2> m_contr2;
    btod_contract2<N1, N2 + K2, K1> m_op1;
    block_tensor<NAB, double> m_ab;
    block_tensor<N3 + K2, double> &m_c;
    double m_kd;
    std::unique_ptr<btod_contract2<N1 + N2, N3, K2> > m_op2;
    btod_contract2<N1 + N2, N3, K2> &second() {
        m_op1.perform(m_ab);
        if (!m_op2) m_op2.reset(new btod_contract2<N1 + N2, N3, K2>(m_contr2, m_ab, 1.0, m_c, 1.0, m_kd));
        return *m_op2;
    }
public:
    btod_contract3(const contraction2<N1, N2 + K2, K1> &contr1, const contraction2<N1 + N2, N3, K2> &contr2,
                   block_tensor<N1 + K1, double> &bta, block_tensor<N2 + K1 + K2, double> &btb,
                   block_tensor<N3 + K2, double> &btc, double kd = 1.0)
        : m_contr2(contr2), m_op1(contr1, bta, btb),
          m_ab(contraction_space(contr1, bta.get_bis(), btb.get_bis())), m_c(btc), m_kd(kd) { }
    void perform(block_tensor<N1 + N2 + N3, double> &btd) override { second().perform(btd); }
    void perform(block_tensor<N1 + N2 + N3, double> &btd, double d) override { second().perform(btd, d); }
};

// direct_block_tensor (libtensor/block_tensor/direct_block_tensor.h:22): a
// block tensor holding an operation's result, computed when an operation
// first reads it, so that it needs no separate perform.  The whole result is
// formed on the device at that first read (the reference forms each block
// when it is requested); refresh() forms it again at the next read, after the
// operation's inputs changed.
template<size_t N>
class direct_block_tensor : public block_tensor<N, double> {
    additive_bto<N> &m_op;
    bool m_ready = false;
public:
    direct_block_tensor(additive_bto<N> &op, const block_index_space<N> &bis)
        : block_tensor<N, double>(bis), m_op(op) { }
    ltg_bt *handle() override {
        if (!m_ready) {
            m_ready = true;                  // the operation's own handle() calls land below
            m_op.perform(*this);
        }
        return block_tensor<N, double>::handle();
    }
    void refresh() { m_ready = false; }
};

}  // namespace libtensor

#endif  // LIBTENSOR_B200_LIBTENSOR_H
