// Host engine implementation; see ltg_host.hpp.
#include "ltg_host.hpp"

#include <algorithm>
#include <atomic>
#include <list>
#include <map>
#include <set>
#include <thread>

namespace ltg {

// ---------------------------------------------------------------- Bis

void Bis::finalize() {
    if (n < 1 || n > kMaxOrder) throw error(kErrBadDims, "tensor order out of range");
    for (int d = 0; d < n; d++) {
        if (dims[d] < 1) throw error(kErrBadDims, "dimension must be positive");
        std::vector<int64_t> &s = starts[d];
        if (s.empty() || s[0] != 0) s.insert(s.begin(), 0);
        for (size_t i = 1; i < s.size(); i++)
            if (s[i] <= s[i - 1] || s[i] >= dims[d])
                throw error(kErrBadDims, "split points must be increasing and inside the dimension");
        bidims[d] = (int64_t)s.size();
    }
}

Bis Bis::permuted(const Perm &p) const {
    Bis r = *this;
    int64_t dd[kMaxOrder]; int tt[kMaxOrder];
    for (int d = 0; d < n; d++) { dd[d] = dims[d]; tt[d] = type[d]; }
    p.apply(dd); p.apply(tt);
    for (int d = 0; d < n; d++) { r.dims[d] = dd[d]; r.type[d] = tt[d]; r.starts[d] = starts[p.p[d]]; r.bidims[d] = bidims[p.p[d]]; }
    return r;
}

bool Bis::equals(const Bis &o) const {
    if (n != o.n) return false;
    for (int d = 0; d < n; d++)
        if (dims[d] != o.dims[d] || starts[d] != o.starts[d]) return false;
    return true;
}

// ---------------------------------------------------------------- labels

bool SeLabel::is_allowed(int n, const int64_t *bidx) const {
    // OR over products; a product holds if every term holds; a term with an
    // unlabelled block is skipped; an empty product fails the whole rule
    // (libtensor/symmetry/inst/se_label_impl.h:74-112).
    for (const std::vector<LabelTerm> &pr : rule) {
        if (pr.empty()) return false;
        bool ok = true;
        for (const LabelTerm &t : pr) {
            if (t.intr < 0) continue;
            int prod = 0;
            bool valid = true;
            for (int d = 0; d < n; d++) {
                if (!t.seq[d]) continue;
                int l = labels[d].empty() ? -1 : labels[d][bidx[d]];
                if (l < 0) { valid = false; break; }
                if (t.seq[d] & 1) prod ^= l;
            }
            if (!valid) continue;
            if (prod != t.intr) { ok = false; break; }
        }
        if (ok) return true;
    }
    return false;
}

// ---------------------------------------------------------------- orbits

namespace {

// Applies symmetry element e (in perm, part, label order) to idx/tr.
// se_part without maps and se_label leave the index unchanged.
inline void apply_perm_elem(const SePerm &e, int n, int64_t *idx, Transf &tr) {
    e.perm.apply(idx);
    Transf t; t.perm = e.perm; t.coeff = e.coeff;
    tr.transform(t);
}

}  // namespace

const Transf *Orbit::find(int64_t aidx) const {
    auto it = std::lower_bound(members.begin(), members.end(), aidx,
        [](const std::pair<int64_t, Transf> &a, int64_t b) { return a.first < b; });
    if (it == members.end() || it->first != aidx) return nullptr;
    return &it->second;
}

void build_orbit(const Bis &bis, const Symmetry &sym, int64_t aidx0, Orbit &o) {
    const int n = bis.n;
    struct Q { int64_t idx[kMaxOrder]; Transf tr; };
    std::vector<std::pair<int64_t, size_t>> orb;   // (abs index, transform slot)
    std::vector<Transf> trs;
    std::vector<Q> q;
    std::vector<Q> t;
    std::vector<std::pair<int64_t, size_t>> can1, can2, merged;
    o.allowed = true;

    Q q0; bis.unabs(aidx0, q0.idx); q0.tr = Transf::identity(n);
    trs.push_back(q0.tr);
    orb.push_back({aidx0, 0});
    q.push_back(q0);
    const size_t nelem = sym.perm.size() + sym.part.size() + sym.label.size();

    while (!q.empty()) {
        Q cur = q.back(); q.pop_back();
        t.clear();
        // Apply every element in insertion order; partition and label
        // elements only contribute allowed-ness.
        for (size_t e = 0; e < nelem; e++) {
            Q nx = cur;
            if (e < sym.perm.size()) {
                apply_perm_elem(sym.perm[e], n, nx.idx, nx.tr);
            } else if (e < sym.perm.size() + sym.part.size()) {
                if (o.allowed) o.allowed = sym.part[e - sym.perm.size()].is_allowed(n, cur.idx);
            } else {
                if (o.allowed) o.allowed = sym.label[e - sym.perm.size() - sym.part.size()].is_allowed(n, cur.idx);
            }
            t.push_back(nx);
        }
        can1.clear();
        for (size_t i = 0; i < t.size(); i++) {
            int64_t a1 = bis.abs(t[i].idx);
            auto it = std::lower_bound(orb.begin(), orb.end(), std::make_pair(a1, (size_t)0),
                [](const std::pair<int64_t, size_t> &x, const std::pair<int64_t, size_t> &y) { return x.first < y.first; });
            if (it == orb.end() || it->first != a1) can1.push_back({a1, i});
        }
        std::stable_sort(can1.begin(), can1.end(),
            [](const std::pair<int64_t, size_t> &x, const std::pair<int64_t, size_t> &y) { return x.first < y.first; });
        can1.erase(std::unique(can1.begin(), can1.end(),
            [](const std::pair<int64_t, size_t> &x, const std::pair<int64_t, size_t> &y) { return x.first == y.first; }), can1.end());
        can2.clear();
        for (auto &c : can1) {
            size_t j = trs.size();
            trs.push_back(t[c.second].tr);
            can2.push_back({c.first, j});
            Q nq; bis.unabs(c.first, nq.idx); nq.tr = trs[j];
            q.push_back(nq);
        }
        merged.resize(orb.size() + can2.size());
        std::merge(orb.begin(), orb.end(), can2.begin(), can2.end(), merged.begin(),
            [](const std::pair<int64_t, size_t> &x, const std::pair<int64_t, size_t> &y) { return x.first < y.first; });
        orb.swap(merged);
    }

    // Transforms are starter -> target; convert to canonical -> target:
    // T(0->i) = [T(s->0) Tinv(s->i)]^-1 (orbit_impl.h:282-297).
    Transf tr0 = trs[orb[0].second];
    o.canonical = orb[0].first;
    o.members.clear();
    o.members.reserve(orb.size());
    for (auto &m : orb) {
        Transf x = trs[m.second];
        x.invert();
        x.transform(tr0);
        x.invert();
        o.members.push_back({m.first, x});
    }
}

void OrbitTable::build(const Bis &bis, const Symmetry &sym) {
    const int64_t nb = bis.nblocks();
    canon.assign(nb, -1);
    tr.assign(nb, Transf::identity(bis.n));
    allowed.assign(nb, 0);
    canon_list.clear();
    Orbit o;
    // Canonical index and allowed flag are starter-independent: fill them per
    // orbit from its minimum.
    for (int64_t a = 0; a < nb; a++) {
        if (canon[a] >= 0) continue;
        build_orbit(bis, sym, a, o);
        for (auto &m : o.members) { canon[m.first] = o.canonical; allowed[m.first] = o.allowed; }
        if (o.allowed) canon_list.push_back(o.canonical);
    }
    std::sort(canon_list.begin(), canon_list.end());
    // The transform canonical -> block is taken from an orbit started at
    // that block, as the pair-list builder does
    // (gen_bto_contract2_clst_builder_impl.h:296-300).
    const bool trivial = sym.perm.empty();
    for (int64_t a = 0; a < nb; a++) {
        if (trivial || canon[a] == a) continue;
        build_orbit(bis, sym, a, o);
        const Transf *t = o.find(a);
        tr[a] = *t;
    }
}

// ---------------------------------------------------------------- directory

void BlockTensorHost::build_directory() {
    orbits.build(bis, sym);
    blk_abs = orbits.canon_list;
    blk_off.resize(blk_abs.size());
    blk_size.resize(blk_abs.size());
    nonzero.assign(blk_abs.size(), 0);
    slot_of.assign(bis.nblocks(), -1);
    int64_t off = 0;
    int64_t bidx[kMaxOrder];
    for (size_t i = 0; i < blk_abs.size(); i++) {
        bis.unabs(blk_abs[i], bidx);
        blk_size[i] = bis.block_size(bidx);
        blk_off[i] = off;
        slot_of[blk_abs[i]] = (int64_t)i;
        // Every block starts on a 32-byte boundary (4 doubles) so vector
        // loads of block-aligned rows stay aligned.
        off += (blk_size[i] + 3) & ~int64_t(3);
    }
    total_elems = off;
}

// ---------------------------------------------------------------- contraction

void Contraction::init(int n, int m, int k, const Perm &pc) {
    N = n; M = m; K = k; permc = pc; nk_set = 0;
    if (n + m + k > kMaxOrder * 3 / 2 || n + k > kMaxOrder || m + k > kMaxOrder || n + m > kMaxOrder)
        throw error(kErrUnsupported, "contraction order too large");
    for (int i = 0; i < 2 * (N + M + K); i++) conn[i] = -1;
    if (K == 0) connect();
}

void Contraction::contract(int ia, int ib) {
    if (nk_set >= K) throw error(kErrBadArg, "contraction is complete");
    if (ia < 0 || ia >= NA() || ib < 0 || ib >= NB()) throw error(kErrBadArg, "contracted index out of range");
    int ja = NC() + ia, jb = NC() + NA() + ib;
    if (conn[ja] != -1 || conn[jb] != -1) throw error(kErrBadArg, "index already contracted");
    conn[ja] = jb; conn[jb] = ja;
    if (++nk_set == K) connect();
}

void Contraction::connect() {
    // Uncontracted A/B slots in slot order, permuted by permc, connect to the
    // C slots (contraction2.h:309-322).
    int64_t connc[kMaxOrder];
    int nc = 0;
    for (int i = NC(); i < 2 * (N + M + K); i++)
        if (conn[i] == -1 || conn[i] < NC()) connc[nc++] = i;
    Perm p = permc; p.n = NC();
    p.apply(connc);
    for (int i = 0; i < NC(); i++) { conn[i] = connc[i]; conn[connc[i]] = i; }
}

void Contraction::make_seqc(int64_t *seqc) const {
    for (int i = 0, j = 0; i < NA() + NB(); i++)
        if (conn[NC() + i] < NC()) seqc[j++] = conn[NC() + i];
}

void Contraction::adjust_permc(const int64_t *s1, const int64_t *s2) {
    // pb[i] = position in s2 of s1[i]; new permc[i] = pb[permc[i]].
    Perm pb = Perm::identity(NC());
    for (int i = 0; i < NC(); i++)
        for (int j = 0; j < NC(); j++)
            if (s2[j] == s1[i]) { pb.p[i] = (int8_t)j; break; }
    Perm r = Perm::identity(NC());
    for (int i = 0; i < NC(); i++) r.p[i] = pb.p[permc.p[i]];
    permc = r;
}

void Contraction::permute_a(const Perm &pa) {
    if (pa.is_identity()) return;
    int64_t seqc1[kMaxOrder], seqc2[kMaxOrder], seqa[kMaxOrder];
    make_seqc(seqc1);
    for (int i = 0; i < NA(); i++) seqa[i] = conn[NC() + i];
    pa.apply(seqa);
    for (int i = 0; i < NA(); i++) { conn[NC() + i] = seqa[i]; conn[seqa[i]] = NC() + i; }
    make_seqc(seqc2);
    adjust_permc(seqc1, seqc2);
}

void Contraction::permute_b(const Perm &pb) {
    if (pb.is_identity()) return;
    int64_t seqc1[kMaxOrder], seqc2[kMaxOrder], seqb[kMaxOrder];
    make_seqc(seqc1);
    for (int i = 0; i < NB(); i++) seqb[i] = conn[NC() + NA() + i];
    pb.apply(seqb);
    for (int i = 0; i < NB(); i++) { conn[NC() + NA() + i] = seqb[i]; conn[seqb[i]] = NC() + NA() + i; }
    make_seqc(seqc2);
    adjust_permc(seqc1, seqc2);
}

void Contraction::permute_c(const Perm &pc) {
    permc.permute(pc);
    connect();
}

// ---------------------------------------------------------------- result space

namespace {

// All elements of the group generated by the perm generators (closure).
std::vector<SePerm> perm_group(int n, const std::vector<SePerm> &gens) {
    std::vector<SePerm> g;
    SePerm id; id.perm = Perm::identity(n); id.coeff = 1.0;
    g.push_back(id);
    for (size_t i = 0; i < g.size(); i++) {
        for (const SePerm &s : gens) {
            SePerm x = g[i];
            x.perm.permute(s.perm);
            x.coeff *= s.coeff;
            bool found = false;
            for (const SePerm &y : g) if (y.perm == x.perm) {
                if (y.coeff != x.coeff)
                    throw error(kErrSymmetry, "inconsistent permutational symmetry (sign)");
                found = true; break;
            }
            if (!found) g.push_back(x);
            if (g.size() > 40320) throw error(kErrUnsupported, "permutation group too large");
        }
    }
    return g;
}

}  // namespace

void contract2_result_space(const Contraction &c, const BlockTensorHost &a,
    const BlockTensorHost &b, Bis &bisc, Symmetry &symc) {
    const int NC = c.NC(), NA = c.NA(), NB = c.NB();
    // Result dims and splits follow the connected argument dims
    // (gen_bto_contract2_bis).
    bisc = Bis();
    bisc.n = NC;
    for (int i = 0; i < NC; i++) {
        int64_t s = c.conn[i];
        const Bis &src = (s < NC + NA) ? a.bis : b.bis;
        int d = (int)((s < NC + NA) ? s - NC : s - NC - NA);
        bisc.dims[i] = src.dims[d];
        bisc.starts[i] = src.starts[d];
        bisc.bidims[i] = src.bidims[d];
    }
    for (int i = 0; i < NC; i++) {
        bisc.type[i] = i;
        for (int j = 0; j < i; j++)
            if (bisc.dims[j] == bisc.dims[i] && bisc.starts[j] == bisc.starts[i]) { bisc.type[i] = bisc.type[j]; break; }
    }
    // Contracted dims must have identical block structure in A and B.
    for (int i = 0; i < NA; i++) {
        int64_t s = c.conn[NC + i];
        if (s >= NC + NA) {
            int j = (int)(s - NC - NA);
            if (a.bis.dims[i] != b.bis.dims[j] || a.bis.starts[i] != b.bis.starts[j])
                throw error(kErrBadDims, "contracted dimensions have different block structure");
        }
    }
    symc = Symmetry();

    // --- permutational symmetry: direct product of the argument groups,
    // set-wise stabilised on the contracted index pairs (a pair may move onto
    // another pair as a whole, outer indices stay outer), restricted to the
    // result (so_dirprod + so_reduce; permutation_group::make_setstabilizer,
    // libtensor/symmetry/inst/permutation_group_impl.h:459-580, and
    // so_reduce_se_perm_impl.h:22-94).
    // Contracted pair number of every A and B dim (-1 for outer dims).
    int kpos_a[kMaxOrder], kpos_b[kMaxOrder];
    {
        int q = 0;
        for (int i = 0; i < NA; i++) {
            kpos_a[i] = -1;
            int64_t s = c.conn[NC + i];
            if (s >= NC + NA) { kpos_a[i] = q; kpos_b[s - NC - NA] = q; q++; }
        }
        for (int j = 0; j < NB; j++)
            if (c.conn[NC + NA + j] < NC) kpos_b[j] = -1;
    }
    struct RElem { Perm pc; double coeff; std::vector<int> sigma; };
    auto restrict_group = [&](const BlockTensorHost &t, int base, int nt, const int *kpos,
                              std::vector<RElem> &out) {
        std::vector<SePerm> g = perm_group(nt, t.sym.perm);
        for (const SePerm &e : g) {
            bool ok = true;
            std::vector<int> sigma(c.K, -1);
            for (int i = 0; i < nt && ok; i++) {
                int src = e.perm.p[i];
                if ((kpos[i] < 0) != (kpos[src] < 0)) ok = false;          // outer <-> contracted
                else if (kpos[i] >= 0) {
                    sigma[kpos[i]] = kpos[src];
                    // the moved dim must have the same block structure
                    if (t.bis.dims[i] != t.bis.dims[src] || t.bis.starts[i] != t.bis.starts[src]) ok = false;
                }
            }
            if (!ok) continue;
            Perm pc = Perm::identity(NC);
            for (int i = 0; i < nt; i++) {
                if (kpos[i] >= 0) continue;
                int r = (int)c.conn[base + i];
                int rsrc = (int)c.conn[base + e.perm.p[i]];
                pc.p[r] = (int8_t)rsrc;
            }
            out.push_back({pc, e.coeff, sigma});
        }
    };
    std::vector<RElem> ga, gb;
    restrict_group(a, NC, NA, kpos_a, ga);
    restrict_group(b, NC + NA, NB, kpos_b, gb);
    std::vector<SePerm> gc;
    for (auto &x : ga) for (auto &y : gb) {
        if (x.sigma != y.sigma) continue;      // pairs must move together
        SePerm e; e.perm = x.pc; e.perm.permute(y.pc); e.coeff = x.coeff * y.coeff;
        if (e.perm.is_identity()) {
            if (e.coeff != 1.0) throw error(kErrSymmetry, "anti-symmetric identity permutation");
            continue;
        }
        bool dup = false;
        for (auto &z : gc) if (z.perm == e.perm) { dup = true; break; }
        if (!dup) gc.push_back(e);
    }
    symc.perm = gc;

    // --- partitions: a result partition is forbidden when every choice of
    // contracted partitions is forbidden in A or in B (so_reduce_se_part,
    // forbidden-only case).
    if (!a.sym.part.empty() || !b.sym.part.empty()) {
        if (a.sym.part.size() > 1 || b.sym.part.size() > 1)
            throw error(kErrUnsupported, "more than one se_part element per tensor");
        const SePart *pa = a.sym.part.empty() ? nullptr : &a.sym.part[0];
        const SePart *pb = b.sym.part.empty() ? nullptr : &b.sym.part[0];
        SePart pcx;
        for (int i = 0; i < NC; i++) {
            int64_t s = c.conn[i];
            const SePart *src = (s < NC + NA) ? pa : pb;
            int d = (int)((s < NC + NA) ? s - NC : s - NC - NA);
            pcx.pdims[i] = src ? src->pdims[d] : 1;
            pcx.bipdims[i] = bisc.bidims[i] / pcx.pdims[i];
        }
        // contracted partition extents (must agree between A and B)
        std::vector<int> ka_dims, kb_dims;
        std::vector<int64_t> kp;
        for (int i = 0; i < NA; i++) {
            int64_t s = c.conn[NC + i];
            if (s < NC + NA) continue;
            int j = (int)(s - NC - NA);
            int64_t p1 = pa ? pa->pdims[i] : 1, p2 = pb ? pb->pdims[j] : 1;
            int64_t p = (p1 == p2) ? p1 : 1;
            if (p1 != p2 && p1 != 1 && p2 != 1)
                throw error(kErrUnsupported, "contracted dims with different partitioning");
            if (p1 != p2) p = std::max(p1, p2);
            ka_dims.push_back(i); kb_dims.push_back(j); kp.push_back(p);
        }
        int64_t npc = 1;
        for (int i = 0; i < NC; i++) npc *= pcx.pdims[i];
        int64_t nkp = 1;
        for (int64_t p : kp) nkp *= p;
        pcx.forbidden.assign(npc, 0);
        bool any = false;
        int64_t pci[kMaxOrder], pai[kMaxOrder], pbi[kMaxOrder];
        for (int64_t x = 0; x < npc; x++) {
            int64_t r = x;
            for (int i = NC - 1; i >= 0; i--) { pci[i] = r % pcx.pdims[i]; r /= pcx.pdims[i]; }
            bool allowed_any = false;
            for (int64_t y = 0; y < nkp && !allowed_any; y++) {
                int64_t ry = y;
                std::vector<int64_t> kv(kp.size());
                for (int q = (int)kp.size() - 1; q >= 0; q--) { kv[q] = ry % kp[q]; ry /= kp[q]; }
                for (int i = 0; i < NA; i++) {
                    int64_t s = c.conn[NC + i];
                    if (s < NC) pai[i] = pci[s];
                }
                for (int j = 0; j < NB; j++) {
                    int64_t s = c.conn[NC + NA + j];
                    if (s < NC) pbi[j] = pci[s];
                }
                for (size_t q = 0; q < kp.size(); q++) {
                    pai[ka_dims[q]] = pa ? (kv[q] * pa->pdims[ka_dims[q]] / kp[q]) : 0;
                    pbi[kb_dims[q]] = pb ? (kv[q] * pb->pdims[kb_dims[q]] / kp[q]) : 0;
                }
                bool fa = false, fb = false;
                if (pa) { int64_t ab = 0; for (int i = 0; i < NA; i++) ab = ab * pa->pdims[i] + (pa->pdims[i] > 1 ? pai[i] : 0); fa = pa->forbidden[ab]; }
                if (pb) { int64_t ab = 0; for (int j = 0; j < NB; j++) ab = ab * pb->pdims[j] + (pb->pdims[j] > 1 ? pbi[j] : 0); fb = pb->forbidden[ab]; }
                if (!fa && !fb) allowed_any = true;
            }
            if (!allowed_any) { pcx.forbidden[x] = 1; any = true; }
        }
        if (any) symc.part.push_back(pcx);
    }

    // --- labels: substitute every label combination of the contracted dims
    // into the argument rules; the result rule is the OR over combinations of
    // the AND of both substituted rules (er_reduce for abelian tables).
    if (!a.sym.label.empty() || !b.sym.label.empty()) {
        if (a.sym.label.size() > 1 || b.sym.label.size() > 1)
            throw error(kErrUnsupported, "more than one se_label element per tensor");
        const SeLabel *la = a.sym.label.empty() ? nullptr : &a.sym.label[0];
        const SeLabel *lb = b.sym.label.empty() ? nullptr : &b.sym.label[0];
        int nirrep = la ? la->nirrep : lb->nirrep;
        if (la && lb && la->nirrep != lb->nirrep) throw error(kErrSymmetry, "label tables differ");
        SeLabel lc;
        lc.nirrep = nirrep;
        for (int i = 0; i < NC; i++) {
            int64_t s = c.conn[i];
            const SeLabel *src = (s < NC + NA) ? la : lb;
            int d = (int)((s < NC + NA) ? s - NC : s - NC - NA);
            if (src && !src->labels[d].empty()) lc.labels[i] = src->labels[d];
            else lc.labels[i].assign(bisc.bidims[i], -1);
        }
        // label sets present on each contracted pair
        std::vector<std::vector<int>> kset;
        std::vector<int> kda, kdb;
        for (int i = 0; i < NA; i++) {
            int64_t s = c.conn[NC + i];
            if (s < NC + NA) continue;
            int j = (int)(s - NC - NA);
            std::set<int> ls;
            const std::vector<int> *v = (la && !la->labels[i].empty()) ? &la->labels[i]
                : (lb && !lb->labels[j].empty()) ? &lb->labels[j] : nullptr;
            if (v) for (int l : *v) ls.insert(l);
            if (!v || ls.count(-1)) ls.insert(-1);
            kset.push_back(std::vector<int>(ls.begin(), ls.end()));
            kda.push_back(i); kdb.push_back(j);
        }
        auto substitute = [&](const SeLabel *l, int base, int nt, const std::vector<int> &kd,
                              const std::vector<int> &kl, std::vector<std::vector<LabelTerm>> &out) {
            // returns the rule of one argument with the contracted labels fixed
            out.clear();
            if (!l) { out.push_back({}); return; }   // no constraint: one empty-but-true marker
            for (const auto &pr : l->rule) {
                std::vector<LabelTerm> np;
                bool prod_ok = true;
                if (pr.empty()) { out.push_back({}); out.back().push_back(LabelTerm()); out.back().back().intr = -2; continue; }
                for (const LabelTerm &t : pr) {
                    if (t.intr < 0) continue;
                    LabelTerm nt_; nt_.intr = t.intr;
                    bool has_outer = false, invalid = false;
                    for (int i = 0; i < nt; i++) {
                        if (!t.seq[i]) continue;
                        int64_t s = c.conn[base + i];
                        if (s < NC) { nt_.seq[s] = t.seq[i]; has_outer = true; }
                        else {
                            size_t q = std::find(kd.begin(), kd.end(), i) - kd.begin();
                            int lab = kl[q];
                            if (lab < 0) invalid = true;
                            else if (t.seq[i] & 1) nt_.intr ^= lab;
                        }
                    }
                    if (invalid) continue;          // unlabelled: term skipped
                    if (!has_outer) {
                        if (nt_.intr != 0) { prod_ok = false; break; }
                        continue;
                    }
                    np.push_back(nt_);
                }
                if (prod_ok) out.push_back(np);
            }
        };
        std::vector<std::vector<LabelTerm>> rule_c;
        std::vector<int> kl(kset.size(), 0);
        std::vector<size_t> pos(kset.size(), 0);
        std::vector<std::vector<LabelTerm>> ra, rb;
        while (true) {
            for (size_t q = 0; q < kset.size(); q++) kl[q] = kset[q][pos[q]];
            substitute(la, NC, NA, kda, kl, ra);
            substitute(lb, NC + NA, NB, kdb, kl, rb);
            for (auto &x : ra) for (auto &y : rb) {
                bool bad = false;
                std::vector<LabelTerm> pr;
                for (auto &t : x) { if (t.intr == -2) bad = true; pr.push_back(t); }
                for (auto &t : y) { if (t.intr == -2) bad = true; pr.push_back(t); }
                if (bad) continue;
                // canonical order for de-duplication
                std::sort(pr.begin(), pr.end(), [&](const LabelTerm &p, const LabelTerm &q) {
                    int c1 = std::memcmp(p.seq, q.seq, kMaxOrder);
                    return c1 != 0 ? c1 < 0 : p.intr < q.intr; });
                pr.erase(std::unique(pr.begin(), pr.end(), [](const LabelTerm &p, const LabelTerm &q) {
                    return std::memcmp(p.seq, q.seq, kMaxOrder) == 0 && p.intr == q.intr; }), pr.end());
                if (pr.empty()) {
                    // unconditional product: every block allowed
                    LabelTerm t; t.intr = -1; pr.push_back(t);
                }
                bool dup = false;
                for (auto &z : rule_c) {
                    if (z.size() != pr.size()) continue;
                    bool same = true;
                    for (size_t u = 0; u < z.size() && same; u++)
                        same = std::memcmp(z[u].seq, pr[u].seq, kMaxOrder) == 0 && z[u].intr == pr[u].intr;
                    if (same) { dup = true; break; }
                }
                if (!dup) rule_c.push_back(pr);
            }
            size_t q = 0;
            for (; q < kset.size(); q++) { if (++pos[q] < kset[q].size()) break; pos[q] = 0; }
            if (q == kset.size()) break;
        }
        lc.rule = rule_c;
        symc.label.push_back(lc);
    }
}

// ---------------------------------------------------------------- schedule

namespace {

// Coalescing of pairs with identical canonical blocks and identical permuted
// contraction (btod_contract2_clst_optimize_impl.h:11-56): for every pair in
// order, the later pairs with the same canonical A and B blocks (the only ones
// that can merge) in order; a pair with the same permuted contraction is added
// into it (coefficient d1 + d2), and when the sum is zero both go.  The same
// result as comparing every pair with every later one, without the quadratic
// scan of the whole list.
void coalesce(const Contraction &c, std::vector<Pair> &v) {
    const size_t n = v.size();
    if (n < 2) return;
    std::vector<uint32_t> order(n);
    for (size_t i = 0; i < n; i++) order[i] = (uint32_t)i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
        return v[x].acia != v[y].acia ? v[x].acia < v[y].acia : v[x].acib < v[y].acib;
    });
    // next later pair with the same canonical blocks
    std::vector<int64_t> next(n, -1);
    for (size_t q = 0; q + 1 < n; q++) {
        const Pair &x = v[order[q]], &y = v[order[q + 1]];
        if (x.acia == y.acia && x.acib == y.acib) next[order[q]] = order[q + 1];
    }
    std::vector<Contraction> conn(n);
    std::vector<char> have(n, 0), alive(n, 1);
    auto conn_of = [&](size_t i) -> const Contraction & {
        if (!have[i]) {
            conn[i] = c;
            conn[i].permute_a(v[i].tra.perm);
            conn[i].permute_b(v[i].trb.perm);
            have[i] = 1;
        }
        return conn[i];
    };
    for (size_t i = 0; i < n; i++) {
        if (!alive[i] || next[i] < 0) continue;
        for (int64_t j = next[i]; j >= 0; j = next[j]) {
            if (!alive[j]) continue;
            if (!conn_of(i).same_conn(conn_of((size_t)j))) continue;
            const double d1 = v[i].tra.coeff * v[i].trb.coeff;
            const double d2 = v[j].tra.coeff * v[j].trb.coeff;
            if (d1 + d2 == 0) {
                alive[i] = alive[j] = 0;
                break;
            }
            v[i].tra.coeff = d1 + d2;
            v[i].trb.coeff = 1.0;
            alive[j] = 0;
        }
    }
    size_t w = 0;
    for (size_t i = 0; i < n; i++)
        if (alive[i]) v[w++] = v[i];
    v.resize(w);
}

}  // namespace

void contract2_schedule(const Contraction &c, const BlockTensorHost &a,
    const BlockTensorHost &b, ContractPlan &plan, int nthreads) {
    plan.contr = c;
    contract2_result_space(c, a, b, plan.bisc, plan.symc);
    OrbitTable oc;
    oc.build(plan.bisc, plan.symc);
    const int NC = c.NC(), NA = c.NA(), NB = c.NB();

    // contracted dims in A order and their partners in B
    int kda[kMaxOrder], kdb[kMaxOrder], nk = 0;
    int64_t kbd[kMaxOrder];
    for (int i = 0; i < NA; i++) {
        int64_t s = c.conn[NC + i];
        if (s >= NC + NA) { kda[nk] = i; kdb[nk] = (int)(s - NC - NA); kbd[nk] = a.bis.bidims[i]; nk++; }
    }
    int64_t nkb = 1;
    for (int q = 0; q < nk; q++) nkb *= kbd[q];

    // unfolded non-zero membership: block present iff its canonical block is
    // stored and non-zero (gen_bto_unfold_block_list)
    auto a_nz = [&](int64_t aidx) {
        int64_t cn = a.orbits.canon[aidx];
        int64_t s = a.slot_of[cn];
        return s >= 0 && a.nonzero[s];
    };
    auto b_nz = [&](int64_t aidx) {
        int64_t cn = b.orbits.canon[aidx];
        int64_t s = b.slot_of[cn];
        return s >= 0 && b.nonzero[s];
    };

    plan.schedule.clear();
    plan.clst.clear();
    plan.flops = 0;
    plan.coalesced = false;
    // Canonical C blocks in chunks over host threads (the reference builds
    // its lists in thread-pool tasks too); chunk results are joined in order,
    // so the schedule is the same for any thread count.
    struct Chunk {
        std::vector<int64_t> schedule;
        std::vector<std::vector<Pair> > clst;
        double flops = 0;
        bool coalesced = false;
    };
    const int64_t ncan = (int64_t)oc.canon_list.size();
    const int64_t per = 64;
    const int64_t nchunks = (ncan + per - 1) / per;
    std::vector<Chunk> chunks((size_t)nchunks);
    auto work = [&](int64_t ci) {
        Chunk &ch = chunks[(size_t)ci];
        int64_t ic[kMaxOrder], ia[kMaxOrder], ib[kMaxOrder], ik[kMaxOrder];
        int64_t da[kMaxOrder], dc[kMaxOrder];
        std::vector<Pair> lst;
        for (int64_t e = ci * per; e < std::min(ncan, (ci + 1) * per); e++) {
            const int64_t cabs = oc.canon_list[(size_t)e];
            plan.bisc.unabs(cabs, ic);
            for (int i = 0; i < NA; i++) { int64_t s = c.conn[NC + i]; if (s < NC) ia[i] = ic[s]; }
            for (int j = 0; j < NB; j++) { int64_t s = c.conn[NC + NA + j]; if (s < NC) ib[j] = ic[s]; }
            lst.clear();
            for (int64_t kk = 0; kk < nkb; kk++) {
                int64_t rr = kk;
                for (int q = nk - 1; q >= 0; q--) { ik[q] = rr % kbd[q]; rr /= kbd[q]; }
                for (int q = 0; q < nk; q++) { ia[kda[q]] = ik[q]; ib[kdb[q]] = ik[q]; }
                int64_t aia = a.bis.abs(ia), aib = b.bis.abs(ib);
                if (!a_nz(aia) || !b_nz(aib)) continue;
                Pair p;
                p.aia = aia; p.acia = a.orbits.canon[aia]; p.tra = a.orbits.tr[aia];
                p.aib = aib; p.acib = b.orbits.canon[aib]; p.trb = b.orbits.tr[aib];
                if (p.tra.perm.n == 0) p.tra.perm.n = NA;
                if (p.trb.perm.n == 0) p.trb.perm.n = NB;
                lst.push_back(p);
            }
            if (lst.empty()) continue;
            const size_t before = lst.size();
            coalesce(c, lst);
            if (lst.size() != before) ch.coalesced = true;
            if (lst.empty()) continue;
            ch.schedule.push_back(cabs);
            ch.clst.push_back(lst);
            plan.bisc.block_dims(ic, dc);
            int64_t csz = 1;
            for (int i = 0; i < NC; i++) csz *= dc[i];
            for (const Pair &p : lst) {
                a.bis.unabs(p.aia, ia);
                a.bis.block_dims(ia, da);
                int64_t kext = 1;
                for (int q = 0; q < nk; q++) kext *= da[kda[q]];
                ch.flops += 2.0 * (double)csz * (double)kext;
            }
        }
    };
    const int nt = (int)std::max<int64_t>(1, std::min<int64_t>(std::max(1, nthreads), nchunks));
    if (nt <= 1) {
        for (int64_t ci = 0; ci < nchunks; ci++) work(ci);
    } else {
        std::atomic<int64_t> nextc(0);
        std::vector<std::thread> pool;
        for (int t = 0; t < nt; t++)
            pool.emplace_back([&]() {
                for (int64_t ci = nextc++; ci < nchunks; ci = nextc++) work(ci);
            });
        for (std::thread &th : pool) th.join();
    }
    for (Chunk &ch : chunks) {
        plan.schedule.insert(plan.schedule.end(), ch.schedule.begin(), ch.schedule.end());
        for (std::vector<Pair> &l : ch.clst) plan.clst.push_back(std::move(l));
        plan.flops += ch.flops;
        plan.coalesced = plan.coalesced || ch.coalesced;
    }
}

// ---------------------------------------------------------------- tasks

namespace {

void fuse(SubDims &s) {
    // drop unit extents, then merge neighbours that are contiguous in both
    // tensors (the loop fusion of contraction2_list_builder).
    SubDims r;
    for (int i = 0; i < s.n; i++) {
        if (s.ext[i] == 1) continue;
        if (r.n > 0) {
            int j = r.n - 1;
            if (r.s0[j] == s.s0[i] * s.ext[i] && r.s1[j] == s.s1[i] * s.ext[i]) {
                r.ext[j] *= s.ext[i];
                r.s0[j] = s.s0[i];
                r.s1[j] = s.s1[i];
                continue;
            }
        }
        if (r.n == kMaxSub) throw error(kErrUnsupported, "too many unfused sub-dimensions");
        r.ext[r.n] = s.ext[i]; r.s0[r.n] = s.s0[i]; r.s1[r.n] = s.s1[i]; r.n++;
    }
    s = r;
}

void rowmajor_strides(int n, const int64_t *d, int64_t *s) {
    int64_t x = 1;
    for (int i = n - 1; i >= 0; i--) { s[i] = x; x *= d[i]; }
}

}  // namespace

void contract2_tasks(const ContractPlan &plan, const BlockTensorHost &a,
    const BlockTensorHost &b, const BlockTensorHost &c, double ka, double kb,
    double kc, std::vector<GemmTask> &tasks, std::vector<CBlockTask> &cblocks) {
    tasks.clear();
    cblocks.clear();
    const int NC = plan.contr.NC(), NA = plan.contr.NA(), NB = plan.contr.NB();
    int64_t ic[kMaxOrder], ia[kMaxOrder], ib[kMaxOrder];
    int64_t dc[kMaxOrder], da[kMaxOrder], db[kMaxOrder];
    int64_t sc[kMaxOrder], sa[kMaxOrder], sb[kMaxOrder];
    for (size_t e = 0; e < plan.schedule.size(); e++) {
        int64_t cabs = plan.schedule[e];
        int64_t cslot = c.slot_of[cabs];
        if (cslot < 0) throw error(kErrState, "result block missing from the output tensor");
        c.bis.unabs(cabs, ic);
        c.bis.block_dims(ic, dc);
        rowmajor_strides(NC, dc, sc);
        CBlockTask cbt;
        cbt.c_off = c.blk_off[cslot];
        cbt.t_begin = (int32_t)tasks.size();
        for (const Pair &p : plan.clst[e]) {
            // Contraction seen from the canonical blocks
            // (gen_bto_contract2_block_impl.h:150-170).
            Contraction ct = plan.contr;
            ct.permute_a(p.tra.perm.inverse());
            ct.permute_b(p.trb.perm.inverse());
            int64_t sa_slot = a.slot_of[p.acia], sb_slot = b.slot_of[p.acib];
            a.bis.unabs(p.acia, ia); a.bis.block_dims(ia, da); rowmajor_strides(NA, da, sa);
            b.bis.unabs(p.acib, ib); b.bis.block_dims(ib, db); rowmajor_strides(NB, db, sb);
            GemmTask t;
            t.c_off = c.blk_off[cslot];
            t.a_off = a.blk_off[sa_slot];
            t.b_off = b.blk_off[sb_slot];
            t.coeff = p.tra.coeff * p.trb.coeff * ka * kb * kc;
            t.cblk = (int32_t)e;
            for (int i = 0; i < NC; i++) {
                int64_t s = ct.conn[i];
                if (s < NC + NA) {
                    int d = (int)(s - NC);
                    if (da[d] != dc[i]) throw error(kErrState, "block extent mismatch (A/C)");
                    t.m.ext[t.m.n] = (int32_t)dc[i]; t.m.s0[t.m.n] = sa[d]; t.m.s1[t.m.n] = sc[i]; t.m.n++;
                } else {
                    int d = (int)(s - NC - NA);
                    if (db[d] != dc[i]) throw error(kErrState, "block extent mismatch (B/C)");
                    t.n.ext[t.n.n] = (int32_t)dc[i]; t.n.s0[t.n.n] = sb[d]; t.n.s1[t.n.n] = sc[i]; t.n.n++;
                }
            }
            for (int i = 0; i < NA; i++) {
                int64_t s = ct.conn[NC + i];
                if (s < NC + NA) continue;
                int j = (int)(s - NC - NA);
                if (da[i] != db[j]) throw error(kErrState, "block extent mismatch (A/B)");
                t.k.ext[t.k.n] = (int32_t)da[i]; t.k.s0[t.k.n] = sa[i]; t.k.s1[t.k.n] = sb[j]; t.k.n++;
            }
            if (tasks.size() == (size_t)cbt.t_begin) {
                // C-side mapping: same m/n linear order, fused on C strides only.
                cbt.cm = t.m; cbt.cn = t.n;
                for (int i = 0; i < cbt.cm.n; i++) cbt.cm.s0[i] = cbt.cm.s1[i];
                for (int i = 0; i < cbt.cn.n; i++) cbt.cn.s0[i] = cbt.cn.s1[i];
                fuse(cbt.cm); fuse(cbt.cn);
                cbt.M = cbt.cm.total(); cbt.N = cbt.cn.total();
                cbt.coeff0 = t.coeff;
            }
            fuse(t.m); fuse(t.n); fuse(t.k);
            cbt.kflops += (double)t.k.total();
            tasks.push_back(t);
        }
        cbt.t_end = (int32_t)tasks.size();
        cblocks.push_back(cbt);
    }
}

// ---------------------------------------------------------------- permuted spaces

void permute_space(const Bis &bis, const Symmetry &sym, const Perm &p, Bis &ob, Symmetry &os) {
    const int n = bis.n;
    ob = bis.permuted(p);
    os = Symmetry();
    Perm pinv = p.inverse();
    for (const SePerm &e : sym.perm) {
        SePerm x; x.perm = Perm::identity(n); x.coeff = e.coeff;
        for (int i = 0; i < n; i++) x.perm.p[i] = pinv.p[e.perm.p[p.p[i]]];
        os.perm.push_back(x);
    }
    for (const SePart &e : sym.part) {
        SePart x;
        for (int d = 0; d < n; d++) { x.pdims[d] = e.pdims[p.p[d]]; x.bipdims[d] = e.bipdims[p.p[d]]; }
        int64_t np = 1;
        for (int d = 0; d < n; d++) np *= x.pdims[d];
        x.forbidden.assign(np, 0);
        int64_t yi[kMaxOrder], xi[kMaxOrder];
        for (int64_t a = 0; a < np; a++) {
            int64_t r = a;
            for (int d = n - 1; d >= 0; d--) { yi[d] = r % x.pdims[d]; r /= x.pdims[d]; }
            for (int d = 0; d < n; d++) xi[p.p[d]] = yi[d];
            int64_t ax = 0;
            for (int d = 0; d < n; d++) ax = ax * e.pdims[d] + xi[d];
            x.forbidden[a] = e.forbidden[ax];
        }
        os.part.push_back(x);
    }
    for (const SeLabel &e : sym.label) {
        SeLabel x;
        x.nirrep = e.nirrep;
        for (int d = 0; d < n; d++) x.labels[d] = e.labels[p.p[d]];
        for (const auto &pr : e.rule) {
            std::vector<LabelTerm> npr;
            for (const LabelTerm &t : pr) {
                LabelTerm u; u.intr = t.intr;
                for (int d = 0; d < n; d++) u.seq[d] = t.seq[p.p[d]];
                npr.push_back(u);
            }
            x.rule.push_back(npr);
        }
        os.label.push_back(x);
    }
}

std::vector<SePerm> perm_group_closure(int n, const std::vector<SePerm> &gens) {
    return perm_group(n, gens);
}

// ---------------------------------------------------------------- transfers

namespace {

void split_units(TransferPlan &plan, int32_t job, int64_t rows, int64_t inner) {
    const int64_t target = 16384;
    int64_t rpu = std::max<int64_t>(1, target / std::max<int64_t>(1, inner));
    for (int64_t r = 0; r < rows; r += rpu) {
        TUnit u; u.job = job; u.pad = 0; u.row_begin = r; u.row_end = std::min(rows, r + rpu);
        plan.units.push_back(u);
    }
}

// Fuses destination dims whose source strides are contiguous for every term.
void fuse_job(TJob &j, TTerm *terms) {
    int nd = 0;
    int32_t ext[kMaxOrder];
    std::vector<std::vector<int32_t>> s(j.nterms, std::vector<int32_t>(kMaxOrder));
    for (int d = 0; d < j.ndim; d++) {
        if (j.ext[d] == 1 && j.ndim > 1) continue;
        if (nd > 0) {
            bool ok = true;
            for (int t = 0; t < j.nterms && ok; t++)
                ok = (int64_t)s[t][nd - 1] == (int64_t)terms[t].sstr[d] * j.ext[d];
            if (ok) {
                ext[nd - 1] *= j.ext[d];
                for (int t = 0; t < j.nterms; t++) s[t][nd - 1] = terms[t].sstr[d];
                continue;
            }
        }
        ext[nd] = j.ext[d];
        for (int t = 0; t < j.nterms; t++) s[t][nd] = terms[t].sstr[d];
        nd++;
    }
    if (nd == 0) { nd = 1; ext[0] = 1; for (int t = 0; t < j.nterms; t++) s[t][0] = 1; }
    j.ndim = nd;
    for (int d = 0; d < kMaxOrder; d++) j.ext[d] = d < nd ? ext[d] : 1;
    for (int t = 0; t < j.nterms; t++)
        for (int d = 0; d < kMaxOrder; d++) terms[t].sstr[d] = d < nd ? s[t][d] : 0;
    j.inner = ext[nd - 1];
}

}  // namespace

void plan_transfer(const std::vector<TransferTerm> &terms, const BlockTensorHost &dst,
                   bool accumulate, TransferPlan &plan) {
    plan = TransferPlan();
    const int n = dst.bis.n;
    if ((int)terms.size() > kMaxTerms_host) throw error(kErrUnsupported, "too many add terms");
    for (const TransferTerm &t : terms) {
        if (t.src->bis.n != n) throw error(kErrBadDims, "operand order differs from the result");
        Bis pb = t.src->bis.permuted(t.perm.inverse());
        // y[d] = x[perm[d]]: dst dim d has the extent of src dim perm[d]
        for (int d = 0; d < n; d++)
            if (t.src->bis.dims[t.perm.p[d]] != dst.bis.dims[d] ||
                t.src->bis.starts[t.perm.p[d]] != dst.bis.starts[d])
                throw error(kErrBadDims, "operand block structure does not match the result");
        (void)pb;
    }
    plan.dst_nonzero.assign(dst.blk_abs.size(), 0);
    int64_t yb[kMaxOrder], xb[kMaxOrder], ext[kMaxOrder], sext[kMaxOrder], sstr[kMaxOrder];
    for (size_t s = 0; s < dst.blk_abs.size(); s++) {
        dst.bis.unabs(dst.blk_abs[s], yb);
        dst.bis.block_dims(yb, ext);
        TJob j;
        j.dst_off = dst.blk_off[s];
        j.ndim = n;
        j.nterms = 0;
        j.term0 = (int32_t)plan.terms.size();
        for (int d = 0; d < kMaxOrder; d++) j.ext[d] = d < n ? (int32_t)ext[d] : 1;
        for (const TransferTerm &t : terms) {
            for (int d = 0; d < n; d++) xb[t.perm.p[d]] = yb[d];
            int64_t xa = t.src->bis.abs(xb);
            if (!t.src->orbits.allowed[xa]) continue;
            int64_t ca = t.src->orbits.canon[xa];
            int64_t cs = t.src->slot_of[ca];
            if (cs < 0 || !t.src->nonzero[cs]) continue;
            const Transf &T = t.src->orbits.tr[xa];
            int64_t cb[kMaxOrder];
            t.src->bis.unabs(ca, cb);
            t.src->bis.block_dims(cb, sext);
            rowmajor_strides(n, sext, sstr);
            TTerm tt;
            tt.src_off = t.src->blk_off[cs];
            tt.coeff = t.coeff * T.coeff;
            tt.src = t.src_index;
            tt.pad = 0;
            for (int d = 0; d < kMaxOrder; d++) tt.sstr[d] = 0;
            for (int d = 0; d < n; d++) {
                int q = T.perm.p[t.perm.p[d]];
                if (sext[q] != ext[d]) throw error(kErrState, "transfer extent mismatch");
                tt.sstr[d] = (int32_t)sstr[q];
            }
            plan.terms.push_back(tt);
            j.nterms++;
        }
        plan.dst_nonzero[s] = j.nterms > 0;
        if (j.nterms == 0 && accumulate) continue;   // nothing to add
        fuse_job(j, plan.terms.data() + j.term0);
        int64_t rows = 1;
        for (int d = 0; d < j.ndim - 1; d++) rows *= j.ext[d];
        plan.bytes += (double)dst.blk_size[s] * 8.0 * (j.nterms + (accumulate ? 2 : 1));
        plan.jobs.push_back(j);
        split_units(plan, (int32_t)plan.jobs.size() - 1, rows, j.inner);
    }
}

void plan_dot(const BlockTensorHost &a, const Perm &pa, const BlockTensorHost &b,
              const Perm &pb, TransferPlan &plan) {
    plan = TransferPlan();
    const int n = a.bis.n;
    if (b.bis.n != n) throw error(kErrBadDims, "dot product operands differ in order");
    Bis ba, bb; Symmetry sa, sb;
    permute_space(a.bis, a.sym, pa, ba, sa);
    permute_space(b.bis, b.sym, pb, bb, sb);
    if (!ba.equals(bb)) throw error(kErrBadDims, "dot product operands differ in block structure");
    // Common group: elements present with the same coefficient in both.
    std::vector<SePerm> ga = perm_group(n, sa.perm), gb = perm_group(n, sb.perm);
    Symmetry common;
    for (const SePerm &x : ga) {
        if (x.perm.is_identity()) continue;
        for (const SePerm &y : gb)
            if (x.perm == y.perm && x.coeff == y.coeff) { common.perm.push_back(x); break; }
    }
    OrbitTable ot;
    ot.build(ba, common);
    int64_t X[kMaxOrder], xb[kMaxOrder], ext[kMaxOrder], sext[kMaxOrder], sstr[kMaxOrder];
    Orbit o;
    for (int64_t xabs : ot.canon_list) {
        ba.unabs(xabs, X);
        ba.block_dims(X, ext);
        // orbit size of X under the common group
        build_orbit(ba, common, xabs, o);
        double weight = (double)o.members.size();
        TJob j;
        j.dst_off = 0;
        j.ndim = n;
        j.nterms = 2;
        j.term0 = (int32_t)plan.terms.size();
        for (int d = 0; d < kMaxOrder; d++) j.ext[d] = d < n ? (int32_t)ext[d] : 1;
        TTerm tt[2];
        bool ok = true;
        for (int w = 0; w < 2 && ok; w++) {
            const BlockTensorHost &t = w == 0 ? a : b;
            const Perm &p = w == 0 ? pa : pb;
            for (int d = 0; d < n; d++) xb[p.p[d]] = X[d];
            int64_t xa = t.bis.abs(xb);
            if (!t.orbits.allowed[xa]) { ok = false; break; }
            int64_t ca = t.orbits.canon[xa];
            int64_t cs = t.slot_of[ca];
            if (cs < 0 || !t.nonzero[cs]) { ok = false; break; }
            const Transf &T = t.orbits.tr[xa];
            int64_t cb[kMaxOrder];
            t.bis.unabs(ca, cb);
            t.bis.block_dims(cb, sext);
            rowmajor_strides(n, sext, sstr);
            tt[w].src_off = t.blk_off[cs];
            tt[w].coeff = T.coeff;
            tt[w].src = w;
            tt[w].pad = 0;
            for (int d = 0; d < kMaxOrder; d++) tt[w].sstr[d] = 0;
            for (int d = 0; d < n; d++) tt[w].sstr[d] = (int32_t)sstr[T.perm.p[p.p[d]]];
        }
        if (!ok) continue;
        tt[0].coeff = tt[0].coeff * tt[1].coeff * weight;
        tt[1].coeff = 1.0;
        plan.terms.push_back(tt[0]);
        plan.terms.push_back(tt[1]);
        fuse_job(j, plan.terms.data() + j.term0);
        int64_t rows = 1;
        for (int d = 0; d < j.ndim - 1; d++) rows *= j.ext[d];
        int64_t nel = 1;
        for (int d = 0; d < n; d++) nel *= ext[d];
        plan.bytes += 16.0 * (double)nel;
        plan.jobs.push_back(j);
        split_units(plan, (int32_t)plan.jobs.size() - 1, rows, j.inner);
    }
}

}  // namespace ltg
