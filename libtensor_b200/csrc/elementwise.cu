// HBM-bound block kernels of the B200 block-tensor path:
//  - permuted, scaled multi-term copy/add over all canonical destination
//    blocks in one launch (replaces tod_copy / tod_add reached through
//    gen_bto_copy and gen_bto_add, libtensor/dense_tensor/impl/tod_copy_impl.h:60-145,
//    libtensor/gen_block_tensor/impl/gen_bto_add_impl.h:128-221);
//  - block-pair dot product with orbit weights and a deterministic two-level
//    FP64 reduction (replaces tod_dotprod through gen_bto_aux_dotprod,
//    libtensor/dense_tensor/impl/tod_dotprod_impl.h:83-150);
//  - scale, seeded fill and orbital-energy denominator.
//
// Every destination block is written exactly once per launch: all terms of
// a btod_add are read in the same pass, so the traffic is (8T + 8) bytes per
// destination element (+8 when accumulating).  A block is traversed as planes
// of A rows x B columns (DJob).  In row mode (every term reads the columns with
// unit stride) each warp takes items of a few thousand elements (a chunk of
// rows x a segment of columns): the outer digits are found once per item with
// 32-bit divisions and shared by all terms, and the lanes walk the item's
// cells (a double, or a double2 where every term is 16-byte aligned) in order,
// stepping row and column without divisions and carrying several cells so that
// several independent loads per term are in flight.  A job with a transposing
// term runs in tiled mode: the CTA stages each tile of a transposing term
// through shared memory, read along the source's contiguous dim and written
// along the destination's.
#include "ltg_device.cuh"

namespace ltg {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
// Cells (one double, or a double2 on the 16-byte path) carried per lane and
// step in row mode: more cells keep more loads in flight, fewer keep the
// registers (and so the resident CTAs) of many-term adds.
template<int NT>
struct CellUnroll { static constexpr int value = NT <= 2 ? 4 : (NT <= 4 ? 2 : 1); };

// Job and term descriptors of the current unit, staged in shared memory.
template<int NT>
struct UnitDesc {
    DJob j;
    DTerm t[NT];
};

// 8-byte asynchronous global -> shared copy (LDGSTS) and the wait for all of
// this thread's outstanding copies.
__device__ __forceinline__ void cp_async8(double *smem, const double *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// Waits for all of this thread's copy groups but the newest (pending = 1) or all.
__device__ __forceinline__ void cp_async_wait_pending(bool one) {
    if (one) asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    else asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

__device__ __forceinline__ void cp_async16(double *smem, const double *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}

template<int NT>
__device__ __forceinline__ void stage_unit(const DJob *__restrict__ jobs, const DTerm *__restrict__ terms,
                                           int32_t job, UnitDesc<NT> &sd) {
    __syncthreads();                              // previous unit done with sd and the tiles
    if (threadIdx.x == 0) sd.j = jobs[job];
    __syncthreads();
    if ((int)threadIdx.x < sd.j.nterms && (int)threadIdx.x < NT) sd.t[threadIdx.x] = terms[sd.j.term0 + threadIdx.x];
    __syncthreads();
}

// Destination and per-term source offsets of row a of plane p.
template<int NT>
__device__ __forceinline__ void plane_row_bases(const UnitDesc<NT> &sd, uint32_t p, uint32_t a,
                                                int64_t &dst, int64_t (&src)[NT]) {
    const DJob &j = sd.j;
    dst = j.dst_off + (int64_t)a * j.dq;
#pragma unroll
    for (int t = 0; t < NT; t++) src[t] = sd.t[t].src_off + (int64_t)a * sd.t[t].sq;
    for (int o = j.nout - 1; o >= 0; o--) {
        const uint32_t e = (uint32_t)j.oext[o];
        const uint32_t q = p / e;
        const uint32_t dig = p - q * e;
        p = q;
        dst += (int64_t)dig * j.odst[o];
#pragma unroll
        for (int t = 0; t < NT; t++) src[t] += (int64_t)dig * sd.t[t].osrc[o];
    }
}

// Row mode: warp item v = (plane, chunk of ra rows, segment of seg columns),
// ordered with the segment fastest; bases advanced to the item's first
// element, extents in na (rows) and nb (columns).
template<int NT>
__device__ __forceinline__ void item_bases(const UnitDesc<NT> &sd, uint32_t v, int64_t &dst,
                                           int64_t (&src)[NT], int &na, int &nb) {
    const DJob &j = sd.j;
    const uint32_t h = v % (uint32_t)j.nseg;
    v /= (uint32_t)j.nseg;
    const uint32_t rc = v % (uint32_t)j.nra;
    const uint32_t p = v / (uint32_t)j.nra;
    const int a0 = (int)rc * j.ra, c0 = (int)h * j.seg;
    na = min(j.ra, j.A - a0);
    nb = min(j.seg, j.B - c0);
    plane_row_bases<NT>(sd, p, (uint32_t)a0, dst, src);
    dst += c0;
#pragma unroll
    for (int t = 0; t < NT; t++) src[t] += (int64_t)c0 * sd.t[t].sb;
}

// Tiled mode: tile v -> plane, first row and column, extents; bases at the
// tile's first row (column 0).
template<int NT>
__device__ __forceinline__ void tile_bases(const UnitDesc<NT> &sd, uint32_t v, int64_t &dst,
                                           int64_t (&src)[NT], int &b0, int &na, int &nb) {
    const DJob &j = sd.j;
    const uint32_t tb = v % (uint32_t)j.ntb;
    v /= (uint32_t)j.ntb;
    const uint32_t ta = v % (uint32_t)j.nta;
    const uint32_t p = v / (uint32_t)j.nta;
    const int ta_ext = (j.A + j.nta - 1) / j.nta, tb_ext = (j.B + j.ntb - 1) / j.ntb;
    const int a0 = (int)ta * ta_ext;
    b0 = (int)tb * tb_ext;
    na = min(ta_ext, j.A - a0);
    nb = min(tb_ext, j.B - b0);
    plane_row_bases<NT>(sd, p, (uint32_t)a0, dst, src);
}

// Tiled mode: per-term constants of the current unit, in registers.
template<int NT>
struct TileTerms {
    const double *src[NT];
    int32_t sq[NT], sb[NT], mode[NT], off[NT], ld[NT], vec[NT];
};

template<int NT>
__device__ __forceinline__ void load_tile_terms(const UnitDesc<NT> &sd, const double *const *srcs,
                                                TileTerms<NT> &tt) {
#pragma unroll
    for (int t = 0; t < NT; t++) {
        const bool on = t < sd.j.nterms;
        tt.src[t] = on ? srcs[sd.t[t].src] : nullptr;
        tt.sq[t] = on ? sd.t[t].sq : 0;
        tt.sb[t] = on ? sd.t[t].sb : 0;
        tt.mode[t] = on ? sd.t[t].tmode : 0;
        tt.off[t] = on ? sd.t[t].toff : 0;
        tt.ld[t] = on ? sd.t[t].tld : 0;
        tt.vec[t] = on ? sd.t[t].tvec : 0;
    }
}

// Issues the copies of every term's tile into shared memory, each along its
// own contiguous direction (columns for layout 0, rows for layout 1; 16-byte
// copies where the term allows), so that all loads of the tile are in flight
// at once.  Offsets inside a tile fit 32 bits (a block holds < 2^31 elements).
// Per-thread positions of the tile mappings for extents (na, nb): threads
// along the columns (da rows apart), along column pairs, or along the rows
// (dc columns apart).  Recomputed only when a tile's extents change.
template<int THREADS>
struct TileMap {
    int na = -1, nb = -1;
    int da, a0, c;           // columns: row step, first row, column
    int vda, va0, vc;        // column pairs
    int dc, c0, ar;          // rows: column step, first column, row
    __device__ __forceinline__ void update(int na_, int nb_) {
        if (na_ == na && nb_ == nb) return;
        na = na_; nb = nb_;
        da = THREADS / nb; a0 = threadIdx.x / nb; c = threadIdx.x - a0 * nb;
        const int ncp = nb >> 1 > 0 ? nb >> 1 : 1;
        vda = THREADS / ncp; va0 = threadIdx.x / ncp; vc = threadIdx.x - va0 * ncp;
        dc = THREADS / na; c0 = threadIdx.x / na; ar = threadIdx.x - c0 * na;
    }
};

template<int NT, int THREADS>
__device__ __forceinline__ void issue_tile(int nt, const TileTerms<NT> &tt, const int64_t (&sbase)[NT],
                                           int b0, int na, int nb, const TileMap<THREADS> &m, double *tiles) {
    // each thread keeps one position along the copied direction and walks
    // the other by pointer increments (threads beyond a whole number of
    // lines stay idle)
#pragma unroll
    for (int t = 0; t < NT; t++) {
        if (t >= nt) break;
        double *T = tiles + tt.off[t];
        const double *src = tt.src[t] + sbase[t] + (int64_t)b0 * tt.sb[t];
        const int sq = tt.sq[t], sb = tt.sb[t], ld = tt.ld[t];
        if (tt.mode[t] == 0) {
            if (tt.vec[t]) {
                if (m.va0 < m.vda) {
                    double *d = T + m.va0 * ld + 2 * m.vc;
                    const double *g = src + (int64_t)m.va0 * sq + 2 * m.vc;
                    for (int a = m.va0; a < na; a += m.vda, d += m.vda * ld, g += (int64_t)m.vda * sq) cp_async16(d, g);
                }
            } else {
                if (m.a0 < m.da) {
                    double *d = T + m.a0 * ld + m.c;
                    const double *g = src + (int64_t)m.a0 * sq + (int64_t)m.c * sb;
                    for (int a = m.a0; a < na; a += m.da, d += m.da * ld, g += (int64_t)m.da * sq) cp_async8(d, g);
                }
            }
        } else {
            if (m.c0 < m.dc) {
                double *d = T + m.c0 * ld + m.ar;
                const double *g = src + (int64_t)m.ar * sq + (int64_t)m.c0 * sb;
                for (int c = m.c0; c < nb; c += m.dc, d += m.dc * ld, g += (int64_t)m.dc * sb) cp_async8(d, g);
            }
        }
    }
}

// One tile of the unit: destination and source bases, first column, extents.
template<int NT>
struct TileGeo {
    int64_t db, sbase[NT];
    int b0, na, nb;
};


// Copy / add: dst = sum_t c_t src_t  or  dst += beta * sum_t c_t src_t, terms
// summed in their order.
template<int NT>
__global__ void __launch_bounds__(kThreads)
transfer_kernel(const DJob *__restrict__ jobs, const DTerm *__restrict__ terms,
                const DUnit *__restrict__ units, int32_t nunits,
                const double *const *__restrict__ srcs, double *__restrict__ dst,
                int32_t accumulate, double beta) {
    constexpr int RU = CellUnroll<NT>::value;
    __shared__ UnitDesc<NT> sd;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const DUnit un = units[u];
        stage_unit<NT>(jobs, terms, un.job, sd);
        const int nt = sd.j.nterms;
        const double *sp[NT];
        double cf[NT];
        int32_t sb[NT], sq[NT];
#pragma unroll
        for (int t = 0; t < NT; t++) {
            sp[t] = t < nt ? srcs[sd.t[t].src] : nullptr;
            cf[t] = t < nt ? sd.t[t].coeff : 0.0;
            sb[t] = t < nt ? sd.t[t].sb : 0;
            sq[t] = t < nt ? sd.t[t].sq : 0;
        }
        // row mode: each warp walks its items cell by cell, lanes consecutive
        const int W = sd.j.vec ? 2 : 1;
        for (int64_t v = un.row_begin + warp; v < un.row_end; v += kWarps) {
            int64_t db, sbase[NT];
            int na, nb;
            item_bases<NT>(sd, (uint32_t)v, db, sbase, na, nb);
            const int ncell = nb / W, ncells = na * ncell;
            const int drow = 32 / ncell, dcol = 32 - drow * ncell;
            int row = lane / ncell, col = lane - row * ncell;
            for (int e0 = 0; e0 < ncells; e0 += 32 * RU) {
                int rr[RU], cc[RU];
                bool ok[RU];
#pragma unroll
                for (int k = 0; k < RU; k++) {
                    ok[k] = e0 + k * 32 + lane < ncells;
                    rr[k] = row;
                    cc[k] = col;
                    row += drow;
                    col += dcol;
                    if (col >= ncell) { col -= ncell; row++; }
                }
                if (W == 2) {
                    double2 val[RU];
#pragma unroll
                    for (int k = 0; k < RU; k++) val[k] = make_double2(0.0, 0.0);
#pragma unroll
                    for (int t = 0; t < NT; t++) {
                        if (t >= nt) break;
#pragma unroll
                        for (int k = 0; k < RU; k++) {
                            if (!ok[k]) continue;
                            const double2 x = *reinterpret_cast<const double2 *>(
                                sp[t] + sbase[t] + (int64_t)rr[k] * sq[t] + 2 * cc[k]);
                            val[k].x += cf[t] * x.x;
                            val[k].y += cf[t] * x.y;
                        }
                    }
#pragma unroll
                    for (int k = 0; k < RU; k++) {
                        if (!ok[k]) continue;
                        double2 *d = reinterpret_cast<double2 *>(dst + db + (int64_t)rr[k] * sd.j.dq + 2 * cc[k]);
                        if (accumulate) {
                            double2 o = *d;
                            o.x = o.x + beta * val[k].x;
                            o.y = o.y + beta * val[k].y;
                            *d = o;
                        } else {
                            *d = val[k];
                        }
                    }
                } else {
                    double val[RU];
#pragma unroll
                    for (int k = 0; k < RU; k++) val[k] = 0.0;
#pragma unroll
                    for (int t = 0; t < NT; t++) {
                        if (t >= nt) break;
#pragma unroll
                        for (int k = 0; k < RU; k++)
                            if (ok[k]) val[k] += cf[t] * sp[t][sbase[t] + (int64_t)rr[k] * sq[t] + (int64_t)cc[k] * sb[t]];
                    }
#pragma unroll
                    for (int k = 0; k < RU; k++) {
                        if (!ok[k]) continue;
                        double *d = dst + db + (int64_t)rr[k] * sd.j.dq + cc[k];
                        if (accumulate) *d = *d + beta * val[k];
                        else *d = val[k];
                    }
                }
            }
        }
    }
}

// Tiled mode (jobs with a transposing term): one CTA per tile at a time; every
// term's tile is staged through shared memory, then combined in term order
// and written along the destination's columns.
constexpr int kTiledThreads = 512;
// Dynamic shared memory of a double-buffered tiled CTA: two CTAs of 512
// threads share an SM, so tiles are double-buffered only while both CTAs'
// sets fit; larger tiles run single-buffered and overlap across the CTAs.
constexpr size_t kTileSmemLimit = 110 * 1024;

// Geometry of the unit's tiles: computed by one thread, two tiles ahead, in
// a ring of three shared slots (current, copies in flight, next).
template<int NT>
__device__ __forceinline__ void geo_ahead(const UnitDesc<NT> &sd, int64_t v, int64_t end, TileGeo<NT> *ring, int slot) {
    if (threadIdx.x == 0 && v < end) {
        TileGeo<NT> &g = ring[slot];
        tile_bases<NT>(sd, (uint32_t)v, g.db, g.sbase, g.b0, g.na, g.nb);
    }
}

template<int NT>
__global__ void __launch_bounds__(kTiledThreads, NT <= 4 ? 2 : 1)
transfer_tiled_kernel(const DJob *__restrict__ jobs, const DTerm *__restrict__ terms,
                      const DUnit *__restrict__ units, int32_t nunits,
                      const double *const *__restrict__ srcs, double *__restrict__ dst,
                      int32_t accumulate, double beta, int32_t stride) {
    __shared__ UnitDesc<NT> sd;
    __shared__ TileGeo<NT> ring[3];
    // one tile per term; two such sets `stride` doubles apart when stride > 0,
    // so that the next tile's copies are in flight while this one is written
    extern __shared__ double tiles[];
    TileMap<kTiledThreads> tm;
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const DUnit un = units[u];
        stage_unit<NT>(jobs, terms, un.job, sd);
        const int nt = sd.j.nterms;
        const int dq = sd.j.dq;
        TileTerms<NT> tt;
        load_tile_terms<NT>(sd, srcs, tt);
        double cf[NT];
#pragma unroll
        for (int t = 0; t < NT; t++) cf[t] = t < nt ? sd.t[t].coeff : 0.0;
        geo_ahead<NT>(sd, un.row_begin, un.row_end, ring, 0);
        geo_ahead<NT>(sd, un.row_begin + 1, un.row_end, ring, 1);
        __syncthreads();
        {
            const TileGeo<NT> &g0 = ring[0];
            tm.update(g0.na, g0.nb);
            issue_tile<NT, kTiledThreads>(nt, tt, g0.sbase, g0.b0, g0.na, g0.nb, tm, tiles);
        }
        cp_async_commit();                                   // the first tile's copies: a group of their own
        int i = 0;
        for (int64_t v = un.row_begin; v < un.row_end; v++, i++) {
            const bool next = v + 1 < un.row_end;
            const TileGeo<NT> &gn = ring[(i + 1) % 3];
            if (stride > 0 && next) {
                tm.update(gn.na, gn.nb);
                issue_tile<NT, kTiledThreads>(nt, tt, gn.sbase, gn.b0, gn.na, gn.nb, tm, tiles + ((i + 1) & 1) * stride);
            }
            cp_async_commit();
            cp_async_wait_pending(stride > 0);               // this tile's copies have landed
            __syncthreads();
            geo_ahead<NT>(sd, v + 2, un.row_end, ring, (i + 2) % 3);
            const double *cur = tiles + (stride > 0 ? (i & 1) * stride : 0);
            const TileGeo<NT> &g = ring[i % 3];
            const int b0 = g.b0, na = g.na, nb = g.nb;
            tm.update(na, nb);
            // a fixed column per thread, rows by pointer increments
            const int da = tm.da, a0 = tm.a0, c = tm.c;
            if (a0 < da) {
                double *d = dst + g.db + b0 + (int64_t)a0 * dq + c;
                const double *p[NT];
                int step[NT];
#pragma unroll
                for (int t = 0; t < NT; t++) {
                    const bool m0 = tt.mode[t] == 0;
                    p[t] = cur + tt.off[t] + (m0 ? a0 * tt.ld[t] + c : c * tt.ld[t] + a0);
                    step[t] = m0 ? da * tt.ld[t] : da;
                }
                for (int a = a0; a < na; a += da, d += (int64_t)da * dq) {
                    double val = 0.0;
#pragma unroll
                    for (int t = 0; t < NT; t++) {
                        if (t >= nt) break;
                        val += cf[t] * *p[t];
                        p[t] += step[t];
                    }
                    if (accumulate) *d = *d + beta * val;
                    else *d = val;
                }
            }
            __syncthreads();                                 // done with this tile's buffer and slot
            if (stride == 0 && next) {
                tm.update(gn.na, gn.nb);
                issue_tile<NT, kTiledThreads>(nt, tt, gn.sbase, gn.b0, gn.na, gn.nb, tm, tiles);
            }
        }
    }
}

__global__ void __launch_bounds__(kTiledThreads, 2)
dot_tiled_kernel(const DJob *__restrict__ jobs, const DTerm *__restrict__ terms,
                 const DUnit *__restrict__ units, int32_t nunits,
                 const double *__restrict__ a, const double *__restrict__ b,
                 double *__restrict__ partials, int32_t stride) {
    __shared__ UnitDesc<2> sd;
    __shared__ TileGeo<2> ring[3];
    __shared__ double red[kTiledThreads];
    extern __shared__ double tiles[];             // as in transfer_tiled_kernel
    TileMap<kTiledThreads> tm;
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const DUnit un = units[u];
        stage_unit<2>(jobs, terms, un.job, sd);
        const double *const ab[2] = {a, b};
        TileTerms<2> tt;
        load_tile_terms<2>(sd, ab, tt);
        double s = 0.0;
        geo_ahead<2>(sd, un.row_begin, un.row_end, ring, 0);
        geo_ahead<2>(sd, un.row_begin + 1, un.row_end, ring, 1);
        __syncthreads();
        {
            const TileGeo<2> &g0 = ring[0];
            tm.update(g0.na, g0.nb);
            issue_tile<2, kTiledThreads>(2, tt, g0.sbase, g0.b0, g0.na, g0.nb, tm, tiles);
        }
        cp_async_commit();
        int it = 0;
        for (int64_t v = un.row_begin; v < un.row_end; v++, it++) {
            const bool next = v + 1 < un.row_end;
            const TileGeo<2> &gn = ring[(it + 1) % 3];
            if (stride > 0 && next) {
                tm.update(gn.na, gn.nb);
                issue_tile<2, kTiledThreads>(2, tt, gn.sbase, gn.b0, gn.na, gn.nb, tm, tiles + ((it + 1) & 1) * stride);
            }
            cp_async_commit();
            cp_async_wait_pending(stride > 0);
            __syncthreads();
            geo_ahead<2>(sd, v + 2, un.row_end, ring, (it + 2) % 3);
            const double *cur = tiles + (stride > 0 ? (it & 1) * stride : 0);
            const TileGeo<2> &g = ring[it % 3];
            const int na = g.na;
            tm.update(na, g.nb);
            const int da = tm.da, a0 = tm.a0, c = tm.c;
            if (a0 < da) {
                const double *p[2];
                int step[2];
#pragma unroll
                for (int t = 0; t < 2; t++) {
                    const bool m0 = tt.mode[t] == 0;
                    p[t] = cur + tt.off[t] + (m0 ? a0 * tt.ld[t] + c : c * tt.ld[t] + a0);
                    step[t] = m0 ? da * tt.ld[t] : da;
                }
                for (int aa = a0; aa < na; aa += da) {
                    s += *p[0] * *p[1];
                    p[0] += step[0];
                    p[1] += step[1];
                }
            }
            __syncthreads();
            if (stride == 0 && next) {
                tm.update(gn.na, gn.nb);
                issue_tile<2, kTiledThreads>(2, tt, gn.sbase, gn.b0, gn.na, gn.nb, tm, tiles);
            }
        }
        red[threadIdx.x] = s;
        __syncthreads();
        for (int w = kTiledThreads / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) partials[u] = red[0] * sd.t[0].coeff;
    }
}

// Dot product: one partial sum per unit (term 0 carries the orbit weight and
// both transform signs), then one fixed-order reduction.
__global__ void __launch_bounds__(kThreads)
dot_kernel(const DJob *__restrict__ jobs, const DTerm *__restrict__ terms,
           const DUnit *__restrict__ units, int32_t nunits,
           const double *__restrict__ a, const double *__restrict__ b,
           double *__restrict__ partials) {
    constexpr int RU = CellUnroll<2>::value;
    __shared__ UnitDesc<2> sd;
    __shared__ double red[kThreads];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const DUnit un = units[u];
        stage_unit<2>(jobs, terms, un.job, sd);
        const double *sp[2] = {sd.t[0].src == 0 ? a : b, sd.t[1].src == 0 ? a : b};
        const int32_t sb[2] = {sd.t[0].sb, sd.t[1].sb}, sq[2] = {sd.t[0].sq, sd.t[1].sq};
        double s = 0.0;
        {
            const int W = sd.j.vec ? 2 : 1;
            for (int64_t v = un.row_begin + warp; v < un.row_end; v += kWarps) {
                int64_t db, sbase[2];
                int na, nb;
                item_bases<2>(sd, (uint32_t)v, db, sbase, na, nb);
                const int ncell = nb / W, ncells = na * ncell;
                const int drow = 32 / ncell, dcol = 32 - drow * ncell;
                int row = lane / ncell, col = lane - row * ncell;
                for (int e0 = 0; e0 < ncells; e0 += 32 * RU) {
                    int rr[RU], cc[RU];
                    bool ok[RU];
#pragma unroll
                    for (int k = 0; k < RU; k++) {
                        ok[k] = e0 + k * 32 + lane < ncells;
                        rr[k] = row;
                        cc[k] = col;
                        row += drow;
                        col += dcol;
                        if (col >= ncell) { col -= ncell; row++; }
                    }
                    if (W == 2) {
#pragma unroll
                        for (int k = 0; k < RU; k++) {
                            if (!ok[k]) continue;
                            const double2 x = *reinterpret_cast<const double2 *>(
                                sp[0] + sbase[0] + (int64_t)rr[k] * sq[0] + 2 * cc[k]);
                            const double2 y = *reinterpret_cast<const double2 *>(
                                sp[1] + sbase[1] + (int64_t)rr[k] * sq[1] + 2 * cc[k]);
                            s += x.x * y.x;
                            s += x.y * y.y;
                        }
                    } else {
#pragma unroll
                        for (int k = 0; k < RU; k++)
                            if (ok[k])
                                s += sp[0][sbase[0] + (int64_t)rr[k] * sq[0] + (int64_t)cc[k] * sb[0]] *
                                     sp[1][sbase[1] + (int64_t)rr[k] * sq[1] + (int64_t)cc[k] * sb[1]];
                    }
                }
            }
        }
        red[threadIdx.x] = s;
        __syncthreads();
        for (int w = kThreads / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) partials[u] = red[0] * sd.t[0].coeff;
    }
}

__global__ void __launch_bounds__(kThreads)
reduce_kernel(const double *__restrict__ partials, int32_t n, double *__restrict__ out) {
    __shared__ double red[kThreads];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += kThreads) s += partials[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

__global__ void scale_kernel(double *__restrict__ x, int64_t n, double c) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t n2 = n / 2;
    double2 *x2 = reinterpret_cast<double2 *>(x);
    for (int64_t k = i; k < n2; k += stride) {
        double2 v = x2[k];
        v.x *= c; v.y *= c;
        x2[k] = v;
    }
    if (i == 0 && (n & 1)) x[n - 1] *= c;
}

// Seeded fill / denominator: one CTA per (block, chunk) unit; element
// coordinates from the block start plus the row-major digits in the block.
__global__ void __launch_bounds__(kThreads)
fill_kernel(double *__restrict__ arena, const int64_t *__restrict__ blk_off,
            const int64_t *__restrict__ blk_start, const int32_t *__restrict__ blk_ext,
            int32_t nblk, int32_t order, DGenGroup g, uint64_t seed, double scale_2m32) {
    for (int b = blockIdx.y; b < nblk; b += gridDim.y) {
        const int32_t *ext = blk_ext + (int64_t)b * kDevMaxOrder;
        const int64_t *st = blk_start + (int64_t)b * kDevMaxOrder;
        int64_t n = 1;
        for (int d = 0; d < order; d++) n *= ext[d];
        for (int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x; e < n;
             e += (int64_t)gridDim.x * kThreads) {
            int64_t x[kDevMaxOrder];
            int64_t r = e;
            for (int d = order - 1; d >= 0; d--) { x[d] = st[d] + r % ext[d]; r /= ext[d]; }
            arena[blk_off[b] + e] = seeded_value(g, seed, scale_2m32, x);
        }
    }
}

__global__ void __launch_bounds__(kThreads)
denom_kernel(double *__restrict__ arena, const int64_t *__restrict__ blk_off,
             const int64_t *__restrict__ blk_start, const int32_t *__restrict__ blk_ext,
             int32_t nblk, const double *__restrict__ eps, const int64_t *__restrict__ eps_off,
             int32_t nocc) {
    for (int b = blockIdx.y; b < nblk; b += gridDim.y) {
        const int32_t *ext = blk_ext + (int64_t)b * kDevMaxOrder;
        const int64_t *st = blk_start + (int64_t)b * kDevMaxOrder;
        int64_t n = (int64_t)ext[0] * ext[1] * ext[2] * ext[3];
        for (int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x; e < n;
             e += (int64_t)gridDim.x * kThreads) {
            int64_t r = e;
            double den = 0.0;
            for (int d = 3; d >= 0; d--) {
                int64_t x = st[d] + r % ext[d];
                r /= ext[d];
                double v = eps[eps_off[d] + x];
                den += d < nocc ? v : -v;
            }
            arena[blk_off[b] + e] /= den;
        }
    }
}

// Doubles between the two tile sets of a double-buffered tiled launch (a
// multiple of 16, keeping 16-byte copies aligned), or 0 when two sets of
// `smem` bytes do not fit.
int32_t tile_stride(size_t smem) {
    const size_t st = (smem / sizeof(double) + 15) / 16 * 16;
    return 2 * st * sizeof(double) <= kTileSmemLimit ? (int32_t)st : 0;
}

int grid_for(int64_t units) {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    int64_t g = units < (int64_t)nsm * 8 ? units : (int64_t)nsm * 8;
    return g < 1 ? 1 : (int)g;
}

template<int NT>
cudaError_t launch_transfer_nt(const DJob *jobs, const DTerm *terms, const DUnit *units, int32_t nrow,
                               int32_t ntiled, size_t smem, const double *const *srcs, double *dst,
                               int32_t accumulate, double beta, cudaStream_t s) {
    if (nrow > 0)
        transfer_kernel<NT><<<grid_for(nrow), kThreads, 0, s>>>(jobs, terms, units, nrow, srcs, dst,
                                                                accumulate, beta);
    if (ntiled > 0) {
        // two tile sets when they fit (double buffering), else one
        const int32_t stride = tile_stride(smem);
        const size_t bytes = stride > 0 ? 2 * (size_t)stride * sizeof(double) : smem;
        if (bytes > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(transfer_tiled_kernel<NT>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
            if (e != cudaSuccess) return e;
        }
        transfer_tiled_kernel<NT><<<grid_for(ntiled), kTiledThreads, bytes, s>>>(
            jobs, terms, units + nrow, ntiled, srcs, dst, accumulate, beta, stride);
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_transfer(const DJob *jobs, const DTerm *terms, const DUnit *units,
                            int32_t nrow, int32_t ntiled, int32_t max_terms, int32_t tile_bytes,
                            const double *const *srcs, double *dst, int32_t accumulate, double beta,
                            cudaStream_t s) {
    if (nrow + ntiled <= 0) return cudaSuccess;
    const size_t smem = (size_t)tile_bytes;
    if (max_terms <= 1) return launch_transfer_nt<1>(jobs, terms, units, nrow, ntiled, smem, srcs, dst, accumulate, beta, s);
    if (max_terms <= 2) return launch_transfer_nt<2>(jobs, terms, units, nrow, ntiled, smem, srcs, dst, accumulate, beta, s);
    if (max_terms <= 4) return launch_transfer_nt<4>(jobs, terms, units, nrow, ntiled, smem, srcs, dst, accumulate, beta, s);
    if (max_terms <= kMaxTerms)
        return launch_transfer_nt<kMaxTerms>(jobs, terms, units, nrow, ntiled, smem, srcs, dst, accumulate, beta, s);
    return cudaErrorInvalidValue;
}

cudaError_t launch_dot(const DJob *jobs, const DTerm *terms, const DUnit *units,
                       int32_t nrow, int32_t ntiled, int32_t tile_bytes, const double *a, const double *b,
                       double *partials, double *out, cudaStream_t s) {
    if (nrow + ntiled <= 0) return cudaMemsetAsync(out, 0, sizeof(double), s);
    if (nrow > 0) dot_kernel<<<grid_for(nrow), kThreads, 0, s>>>(jobs, terms, units, nrow, a, b, partials);
    if (ntiled > 0) {
        const size_t smem = (size_t)tile_bytes;
        const int32_t stride = tile_stride(smem);
        const size_t bytes = stride > 0 ? 2 * (size_t)stride * sizeof(double) : smem;
        if (bytes > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(dot_tiled_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
            if (e != cudaSuccess) return e;
        }
        dot_tiled_kernel<<<grid_for(ntiled), kTiledThreads, bytes, s>>>(jobs, terms, units + nrow, ntiled, a, b,
                                                                          partials + nrow, stride);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    reduce_kernel<<<1, kThreads, 0, s>>>(partials, nrow + ntiled, out);
    return cudaGetLastError();
}

cudaError_t launch_scale(double *x, int64_t n, double c, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    scale_kernel<<<grid_for((n / 2 + kThreads - 1) / kThreads + 1), kThreads, 0, s>>>(x, n, c);
    return cudaGetLastError();
}

cudaError_t launch_fill_seeded(double *arena, const int64_t *blk_off, const int64_t *blk_start,
                               const int32_t *blk_ext, int32_t nblk, int32_t order,
                               const DGenGroup &g, uint64_t seed, double scale_2m32,
                               cudaStream_t s) {
    if (nblk <= 0) return cudaSuccess;
    dim3 grid(64, nblk < 65535 ? nblk : 65535);
    fill_kernel<<<grid, kThreads, 0, s>>>(arena, blk_off, blk_start, blk_ext, nblk, order, g, seed,
                                          scale_2m32);
    return cudaGetLastError();
}

cudaError_t launch_denominator(double *arena, const int64_t *blk_off, const int64_t *blk_start,
                               const int32_t *blk_ext, int32_t nblk, const double *eps,
                               const int64_t *eps_off, int32_t nocc, cudaStream_t s) {
    if (nblk <= 0) return cudaSuccess;
    dim3 grid(64, nblk < 65535 ? nblk : 65535);
    denom_kernel<<<grid, kThreads, 0, s>>>(arena, blk_off, blk_start, blk_ext, nblk, eps, eps_off,
                                           nocc);
    return cudaGetLastError();
}

}  // namespace ltg
