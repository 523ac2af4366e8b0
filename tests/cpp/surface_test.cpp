// Exercises the C++ operator surface (include/libtensor_b200/libtensor.h) the
// way a libtensor user writes the ladder contraction
//   r(i,j,a,b) = 0.5 * sum_cd t(i,j,c,d) V(a,b,c,d)
// on o = 10 (5 per spin), v = 40 (16 + 4 per spin), antisymmetric pairs and
// spin partitions (the pattern of tests/block_tensor/btod_contract2_test.C).
//
//   surface_test schedule        host only: prints the non-zero C blocks
//   surface_test compute FILE    on GPU 0: seeded inputs, contraction, copy,
//                                add and dot products; writes the results to FILE
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "libtensor_b200/libtensor.h"

using namespace libtensor;

namespace {

// POSIX declares a function index() in the global namespace
using libtensor::index;

// splits of a dim holding alpha blocks then beta blocks
template<size_t N>
void split_spin(block_index_space<N> &bis, const mask<N> &m, const std::vector<size_t> &per_spin) {
    std::vector<size_t> sizes(per_spin);
    sizes.insert(sizes.end(), per_spin.begin(), per_spin.end());
    size_t pos = 0;
    for (size_t k = 0; k + 1 < sizes.size(); k++) {
        pos += sizes[k];
        bis.split(m, pos);
    }
}

// antisymmetry in (0,1) and (2,3); spin partitions with the number of beta
// indices in (0,1) equal to that in (2,3)
void add_symmetry(block_tensor<4, double> &bt, const block_index_space<4> &bis) {
    block_tensor_ctrl<4, double> ctrl(bt);
    symmetry<4, double> &sym = ctrl.req_symmetry();
    permutation<4> p01, p23;
    p01.permute(0, 1);
    p23.permute(2, 3);
    sym.insert(se_perm<4, double>(p01, scalar_transf<double>(-1.0)));
    sym.insert(se_perm<4, double>(p23, scalar_transf<double>(-1.0)));
    mask<4> all;
    for (size_t i = 0; i < 4; i++) all[i] = true;
    se_part<4, double> part(bis, all, 2);
    for (size_t x = 0; x < 16; x++) {
        index<4> p;
        for (size_t i = 0; i < 4; i++) p[i] = (x >> (3 - i)) & 1;
        if (p[0] + p[1] != p[2] + p[3]) part.mark_forbidden(p);
    }
    sym.insert(part);
}

block_index_space<4> make_bis(size_t d0, size_t d2, const std::vector<size_t> &s0, const std::vector<size_t> &s2) {
    index<4> i1;
    i1[0] = d0 - 1; i1[1] = d0 - 1; i1[2] = d2 - 1; i1[3] = d2 - 1;
    block_index_space<4> bis(dimensions<4>(index_range<4>(index<4>(), i1)));
    mask<4> m01, m23;
    m01[0] = m01[1] = true;
    m23[2] = m23[3] = true;
    split_spin(bis, m01, s0);
    split_spin(bis, m23, s2);
    return bis;
}

block_index_space<2> make_bis2(size_t d, const std::vector<size_t> &s) {
    index<2> i1;
    i1[0] = d - 1; i1[1] = d - 1;
    block_index_space<2> bis(dimensions<2>(index_range<2>(index<2>(), i1)));
    mask<2> m;
    m[0] = m[1] = true;
    split_spin(bis, m, s);
    return bis;
}

// largest |x - f y| over the canonical blocks of x (same index space; block
// sizes from the device tensor, which may hold a permuted space)
template<size_t N>
double max_diff(block_tensor<N, double> &x, block_tensor<N, double> &y, double f) {
    block_tensor_ctrl<N, double> cx(x), cy(y);
    double m = 0.0;
    for (const index<N> &b : cx.req_canonical_blocks()) {
        int64_t bi[N], bd[N];
        for (size_t k = 0; k < N; k++) bi[k] = (int64_t)b[k];
        b200::check(ltg_bt_block_dims(x.handle(), bi, bd));
        size_t n = 1;
        for (size_t k = 0; k < N; k++) n *= (size_t)bd[k];
        std::vector<double> u(n), w(n);
        cx.get_block(b, u.data());
        cy.get_block(b, w.data());
        for (size_t k = 0; k < u.size(); k++) m = std::max(m, std::fabs(u[k] - f * w[k]));
    }
    return m;
}

}  // namespace

int main(int argc, char **argv) {
    using libtensor::index;
    if (argc < 2) {
        std::fprintf(stderr, "usage: surface_test schedule | compute FILE\n");
        return 2;
    }
    const std::string mode = argv[1];
    try {
        if (mode == "schedule") b200::set_device(-1);
        const std::vector<size_t> occ = {5}, vir = {16, 4};
        block_index_space<4> bis_t = make_bis(10, 40, occ, vir), bis_v = make_bis(40, 40, vir, vir);
        block_tensor<4, double> t(bis_t), v(bis_v);
        add_symmetry(t, bis_t);
        add_symmetry(v, bis_v);
        contraction2<2, 2, 2> contr;
        contr.contract(2, 2);
        contr.contract(3, 3);
        if (mode == "schedule") {
            block_tensor_ctrl<4, double>(t).mark_nonzero();
            block_tensor_ctrl<4, double>(v).mark_nonzero();
            btod_contract2<2, 2, 2> op(contr, t, 1.0, v, 1.0, 0.5);
            for (int64_t a : op.get_schedule()) std::printf("%lld\n", (long long)a);
            return 0;
        }
        if (mode != "compute" || argc < 3) throw bad_parameter("unknown mode");
        block_tensor_ctrl<4, double>(t).fill_seeded(11, 0.01);
        block_tensor_ctrl<4, double>(v).fill_seeded(23, 1.0);
        btod_contract2<2, 2, 2> op(contr, t, 1.0, v, 1.0, 0.5);
        block_index_space<4> bis_r = make_bis(10, 40, occ, vir);
        block_tensor<4, double> r(bis_r);
        op.perform(r);

        // copy with a permutation, a two-term add and dot products: checked
        // through <tp,tp> = 0.25 <t,t> and <t,s> = 1.25 <t,t>
        permutation<4> p0213;
        p0213.permute(1, 2);
        block_tensor<4, double> tp(bis_t);      // takes the permuted space on assignment
        btod_copy<4>(t, p0213, -0.5).perform(tp);
        block_tensor<4, double> s(bis_t);
        add_symmetry(s, bis_t);
        btod_add<4> add(t, 1.0);
        add.add_op(t, 0.25);
        add.perform(s);
        const double dot_tt = btod_dotprod<4>(t, t).calculate();
        const double dot_ts = btod_dotprod<4>(t, s).calculate();
        const double dot_pp = btod_dotprod<4>(tp, tp).calculate();

        // the letter interface: the same operations written as expressions,
        // against the operations written out
        letter i, j, a, b, c1, d1;
        block_tensor<4, double> rl(bis_r), ra(bis_r);
        rl(i|j|a|b) = 0.5 * contract(c1|d1, t(i|j|c1|d1), v(a|b|c1|d1));
        add_symmetry(ra, bis_r);
        ra(i|j|a|b) = r(i|j|a|b) - r(j|i|a|b);                // = 2 r (r is antisymmetric in i, j)
        const double dl_tt = dot_product(t(i|j|a|b), t(i|j|a|b));
        const double dl_tp = dot_product(t(i|j|a|b), t(j|i|a|b));   // = -<t,t>
        block_index_space<2> bis_f = make_bis2(40, vir);
        block_tensor<2, double> fl(bis_f), fe(bis_f);
        fl(a|b) = contract(i|j|c1, t(i|j|a|c1), t(i|j|b|c1));
        contraction2<1, 1, 3> c3;
        c3.contract(0, 0);
        c3.contract(1, 1);
        c3.contract(3, 3);
        btod_contract2<1, 1, 3>(c3, t, t).perform(fe);
        block_tensor<4, double> gl(bis_r), ge(bis_r);
        gl(i|j|a|b) = contract(c1, t(i|j|a|c1), fl(c1|b));
        contraction2<3, 1, 1> c1c;
        c1c.contract(3, 0);
        btod_contract2<3, 1, 1>(c1c, t, fe).perform(ge);
        block_tensor<4, double> hl(bis_r);
        add_symmetry(hl, bis_r);
        hl(i|j|a|b) = r(i|j|a|b);
        hl(i|j|a|b) -= 0.5 * r(i|j|a|b);                      // = r / 2
        // symmetrizers: symm over a pair of index pairs, asymm of a contraction
        // against btod_symmetrize2 of the contraction written out
        block_tensor<4, double> ys(bis_r), gs(bis_r), gse(bis_r);
        add_symmetry(ys, bis_r);
        ys(i|j|a|b) = symm(i|a, j|b, r(i|j|a|b));             // = 2 r
        gs(i|j|a|b) = asymm(a, b, contract(c1, t(i|j|a|c1), fl(c1|b)));
        btod_symmetrize2<4>(ge, 2, 3, false).perform(gse);
        // the same symmetrizer over the contraction itself: both terms written
        // by the contraction's epilogue, no temporary
        block_tensor<4, double> gsf(bis_r), gsm(bis_r);
        btod_contract2<3, 1, 1> gop(c1c, t, fe);
        btod_symmetrize2<4>(gop, 2, 3, false).perform(gsf);
        // and with the contraction in the modular split-precision mode (the
        // recombination adds each element to both terms)
        btod_contract2<3, 1, 1> gopm(c1c, t, fe);
        gopm.set_split_precision(LTG_MODE_OZAKI_CRT, 13);
        btod_symmetrize2<4>(gopm, 2, 3, false).perform(gsm);
        // intermediates: a contraction of a contraction, a contraction of a sum
        // (terms with the same symmetry, and with a spin-only term, whose sum
        // keeps only the common symmetry), the result on the right-hand side,
        // a dot product of a sum -- against the operations written out
        block_tensor<4, double> nl(bis_r), ne(bis_r);
        nl(i|j|a|b) = contract(c1, contract(d1, t(i|j|a|d1), fl(d1|c1)), fl(c1|b));
        btod_contract2<3, 1, 1>(c1c, ge, fe).perform(ne);
        block_tensor<4, double> ql(bis_r), qe(bis_r), u(bis_t);
        add_symmetry(u, bis_t);
        ql(i|j|a|b) = contract(c1, t(i|j|a|c1) + s(i|j|a|c1), fl(c1|b));
        btod_add<4> tu(t, 1.0);
        tu.add_op(s, 1.0);
        tu.perform(u);
        btod_contract2<3, 1, 1>(c1c, u, fe).perform(qe);
        block_tensor<4, double> w(bis_t), wl(bis_r), we(bis_r), uw(bis_t);
        {
            block_tensor_ctrl<4, double> cw(w);
            symmetry<4, double> &sym = cw.req_symmetry();
            mask<4> all;
            for (size_t k = 0; k < 4; k++) all[k] = true;
            se_part<4, double> part(bis_t, all, 2);
            for (size_t x = 0; x < 16; x++) {
                index<4> pp;
                for (size_t k = 0; k < 4; k++) pp[k] = (x >> (3 - k)) & 1;
                if (pp[0] + pp[1] != pp[2] + pp[3]) part.mark_forbidden(pp);
            }
            sym.insert(part);
            cw.fill_seeded(29, 0.01);
            block_tensor_ctrl<4, double> cu(uw);
            cu.req_symmetry().insert(part);
        }
        wl(i|j|a|b) = contract(c1, t(i|j|a|c1) - 2.0 * w(i|j|a|c1), fl(c1|b));
        btod_add<4> twu(t, 1.0);
        twu.add_op(w, -2.0);
        twu.perform(uw);
        btod_contract2<3, 1, 1>(c1c, uw, fe).perform(we);
        block_tensor<4, double> hr(bis_r);
        hr(i|j|a|b) = r(i|j|a|b);
        hr(i|j|a|b) = hr(i|j|a|b) + r(i|j|a|b);               // = 2 r
        const double dl_sum = dot_product(t(i|j|a|b) + s(i|j|a|b), t(i|j|a|b));   // = <t,t> + <s,t>
        // one assignment with intermediates kept and replayed as one graph
        block_tensor<4, double> qg(bis_r);
        b200::assignment<4> asg(qg(i|j|a|b), contract(c1, t(i|j|a|c1) + s(i|j|a|c1), fl(c1|b)));
        asg.capture();
        block_tensor_ctrl<4, double>(qg).fill_seeded(8, 1.0);
        asg.run();
        b200::synchronize();
        const double asg_diff = max_diff(qg, ql, 1.0);
        // a three-tensor contraction and a direct block tensor as an operand,
        // against the two contractions written out:
        //   D(i,j,k,l) = 1/4 sum_ab [sum_cd t(i,j,c,d) v(a,b,c,d)] t(k,l,a,b)
        contraction2<2, 2, 2> cA, cB;
        cA.contract(2, 2);
        cA.contract(3, 3);
        cB.contract(2, 2);
        cB.contract(3, 3);
        block_index_space<4> bis_d = make_bis(10, 10, occ, occ);
        block_tensor<4, double> abx(bis_r), dx(bis_d), d3(bis_d), d4(bis_d);
        btod_contract2<2, 2, 2>(cA, t, v).perform(abx);
        btod_contract2<2, 2, 2>(cB, abx, 1.0, t, 1.0, 0.25).perform(dx);
        btod_contract3<2, 0, 2, 2, 2> c3op(cA, cB, t, v, t, 0.25);
        c3op.perform(d3);
        btod_contract2<2, 2, 2> first(cA, t, v);
        direct_block_tensor<4> dab(first, bis_r);
        btod_contract2<2, 2, 2>(cB, dab, 1.0, t, 1.0, 0.25).perform(d4);
        const double c3_diff = std::max(max_diff(d3, dx, 1.0), max_diff(d4, dx, 1.0));
        // one CUDA graph of the contraction, the permuted copy and the add:
        // run once, captured, inputs overwritten, replayed
        block_tensor<4, double> r2(bis_r), tp2(bis_t), s2(bis_t);
        add_symmetry(s2, bis_t);
        btod_copy<4> cp(t, p0213, -0.5);
        op.perform(r2);
        cp.perform(tp2);
        add.perform(s2);
        b200::begin_capture();
        op.perform(r2);
        cp.perform(tp2);
        add.perform(s2);
        b200::graph g = b200::end_capture();
        block_tensor_ctrl<4, double>(r2).fill_seeded(5, 1.0);
        block_tensor_ctrl<4, double>(tp2).fill_seeded(6, 1.0);
        block_tensor_ctrl<4, double>(s2).fill_seeded(7, 1.0);
        g.launch();
        b200::synchronize();
        const double graph_diff = std::max(max_diff(r2, r, 1.0),
                                           std::max(max_diff(tp2, tp, 1.0), max_diff(s2, s, 1.0)));
        const double diffs[] = {max_diff(rl, r, 1.0), max_diff(ra, r, 2.0),
                                std::fabs(dl_tt - dot_tt), std::fabs(dl_tp + dot_tt),
                                max_diff(fl, fe, 1.0), max_diff(gl, ge, 1.0),
                                max_diff(hl, r, 0.5), max_diff(ys, r, 2.0),
                                max_diff(gse, gs, 1.0), graph_diff,
                                max_diff(nl, ne, 1.0), max_diff(ql, qe, 1.0), max_diff(wl, we, 1.0),
                                max_diff(r, hr, 0.5), std::fabs(dl_sum - dot_tt - dot_ts), asg_diff,
                                (double)asg.operations(), c3_diff, max_diff(gsf, gse, 1.0),
                                max_diff(gsm, gse, 1.0)};

        // the contraction's non-zero blocks in index order, then the dot products
        FILE *f = std::fopen(argv[2], "wb");
        if (!f) throw bad_parameter("cannot open output file");
        block_tensor_ctrl<4, double> c(r);
        const std::vector<index<4> > blocks = c.req_nonzero_blocks();
        std::fprintf(f, "%zu\n", blocks.size());
        for (const index<4> &b : blocks) {
            const dimensions<4> d = bis_r.get_block_dims(b);
            std::vector<double> data(d.get_size());
            c.get_block(b, data.data());
            std::fprintf(f, "%zu %zu %zu %zu %zu\n", b[0], b[1], b[2], b[3], data.size());
            for (double x : data) std::fprintf(f, "%.17g\n", x);
        }
        std::fprintf(f, "%.17g %.17g %.17g\n", dot_tt, dot_ts, dot_pp);
        for (double x : diffs) std::fprintf(f, "%.17g ", x);
        std::fprintf(f, "\n");
        std::fclose(f);
        std::printf("ok %zu blocks, flops %.6g\n", op.get_schedule().size(), op.get_flops());
    } catch (const libtensor::exception &e) {
        std::fprintf(stderr, "libtensor exception: %s\n", e.what());
        return 1;
    }
    return 0;
}
