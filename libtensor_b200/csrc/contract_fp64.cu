// Plain FP64 grouped block-pair contraction on the B200 FP64 tensor path
// (mma.sync m16n8k8 .f64, "DMMA").
//
// Replaces, for every non-zero canonical C block of a btod_contract2
// schedule, the per-block tod_contract2 call chain
// (libtensor/dense_tensor/impl/tod_contract2_impl.h:104-393): the perma/permb
// staging copies, the dgemm (linalg_cblas_level3.C:18-58) and the permc
// permute-add.  One persistent launch walks all (C block, m-tile, n-tile)
// work items from a work queue; each work item accumulates every coalesced
// pair of its C block in registers, so there are no temporaries and no
// atomics, and every C element is written once.
//
// The index permutation of a pair is folded into the tile loader: the
// element (m, k) of the matricised A block lives at
//   a_off + sum_i digit_i(m) * ma_str[i] + sum_j digit_j(k) * ka_str[j]
// (mixed-radix digits over the fused sub-dimensions), computed once per tile
// row and once per k column per stage, and copied with cp.async (zero-filled
// outside the block); 16-byte copies when the pair's k run is contiguous and
// even-aligned, 8-byte copies otherwise.
//
// Fragment k order: the m16n8k8 f64 fragment holds k-slots (t, t+4) of A
// row g and of B column g in lane (g, t).  Any consistent relabelling of the
// 8 k values gives the same sum, so slot t carries k = 2t and slot t+4
// carries k = 2t+1: both operands then read one 16-byte shared-memory word
// per fragment register pair, from a tile stored in natural k order.
#include "ltg_device.cuh"

namespace ltg {
namespace {

__device__ __forceinline__ int64_t mixed_offset(int32_t lin, int n, const int32_t *ext,
                                                const int32_t *str) {
    int64_t off = 0;
    for (int i = n - 1; i >= 0; i--) {
        int32_t e = ext[i];
        int32_t q = lin / e;
        off += (int64_t)(lin - q * e) * str[i];
        lin = q;
    }
    return off;
}

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool pred) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    int sz = pred ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" :: "r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool pred) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    int sz = pred ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" :: "r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template<int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" :: "n"(N)); }

__device__ __forceinline__ void dmma_16x8x8(double *d, const double *a, const double *b) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}
// m16n8k16 (sm_90 and later): the A fragment is the two m16n8k8 fragments of
// k 0-7 and 8-15 one after the other (registers a0-a3, a4-a7), the B
// fragment likewise (b0-b1, b2-b3).
// m8n8k4: lane (g, t) holds A[g][t], B[t][g] (k = t) and C[g][2t], C[g][2t+1].
__device__ __forceinline__ void dmma_8x8x4(double *d, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1]) : "d"(a), "d"(b));
}
__device__ __forceinline__ void dmma_16x8x16(double *d, const double *a0, const double *a1, const double *b0,
                                             const double *b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a0[0]), "d"(a0[1]), "d"(a0[2]), "d"(a0[3]), "d"(a1[0]), "d"(a1[1]), "d"(a1[2]), "d"(a1[3]),
          "d"(b0[0]), "d"(b0[1]), "d"(b1[0]), "d"(b1[1]));
}

// DMMA instruction shapes of a tile configuration
constexpr int kMma16x8x8 = 0, kMma16x8x16 = 1, kMma8x8x4 = 2;

template<int BM_, int BN_, int BK_, int WM_, int WN_, int STAGES_, int MMA_ = kMma16x8x8, int MINB_ = 1>
struct TileCfg {
    static constexpr int BM = BM_, BN = BN_, BK = BK_, WM = WM_, WN = WN_, STAGES = STAGES_;
    static constexpr int MMA = MMA_, MINB = MINB_;     // DMMA shape, CTAs per SM the registers allow
    static constexpr bool K16 = MMA == kMma16x8x16;     // one m16n8k16 DMMA per two k8 steps
    static constexpr int kWarpsM = BM / WM, kWarpsN = BN / WN;
    static constexpr int kThreads = kWarpsM * kWarpsN * 32;
    // padded row stride in doubles: conflict-free 16-byte fragment reads
    // (rows 64 bytes apart mod 128) or 8-byte reads (rows 32 bytes apart)
    static constexpr int kLd = MMA == kMma8x8x4 ? BK + 4 : BK + 8;
    // accumulator fragment: rows per fragment (16 or 8) and doubles per lane
    static constexpr int kFragRows = MMA == kMma8x8x4 ? 8 : 16, kQ = MMA == kMma8x8x4 ? 2 : 4;
    static constexpr int kMT = WM / kFragRows, kNT = WN / 8;
    static constexpr int kStageA = BM * kLd, kStageB = BN * kLd;
    static constexpr size_t kSmem = (size_t)STAGES * (kStageA + kStageB) * sizeof(double)
                                  + (size_t)(BM + BN) * sizeof(int64_t);
    static_assert(kThreads % BK == 0 && kThreads % (BK / 2) == 0, "loader assumes a fixed k column per thread");
    static_assert(BM % WM == 0 && BN % WN == 0 && WM % kFragRows == 0 && WN % 8 == 0, "warp tiling");
    static_assert(BK % 8 == 0, "k step");
};

// Copies the (rows x BK) slab starting at k0 of one operand into shared
// memory.  rowoff[r] < 0 marks rows outside the block (zero fill).
template<class C, int ROWS>
__device__ __forceinline__ void load_operand(double *s, const int64_t *rowoff,
    const double *__restrict__ G, int k0, int K, int nk, const int32_t *kext,
    const int32_t *kstr, bool vec16) {
    const int tid = threadIdx.x;
    if (vec16) {
        constexpr int kCols = C::BK / 2;
        constexpr int kRowsPerPass = C::kThreads / kCols;
        const int kk = (tid % kCols) * 2;
        const int k = k0 + kk;
        const bool kin = k < K;          // K is even on this path
        const int64_t ko = kin ? mixed_offset(k, nk, kext, kstr) : 0;
#pragma unroll
        for (int r0 = 0; r0 < ROWS; r0 += kRowsPerPass) {
            int r = r0 + tid / kCols;
            if (ROWS % kRowsPerPass != 0 && r >= ROWS) break;
            int64_t ro = rowoff[r];
            bool p = kin && ro >= 0;
            cp_async16(&s[r * C::kLd + kk], p ? (const void *)(G + ro + ko) : (const void *)G, p);
        }
    } else {
        constexpr int kRowsPerPass = C::kThreads / C::BK;
        const int kk = tid % C::BK;
        const int k = k0 + kk;
        const bool kin = k < K;
        const int64_t ko = kin ? mixed_offset(k, nk, kext, kstr) : 0;
#pragma unroll
        for (int r0 = 0; r0 < ROWS; r0 += kRowsPerPass) {
            int r = r0 + tid / C::BK;
            if (ROWS % kRowsPerPass != 0 && r >= ROWS) break;
            int64_t ro = rowoff[r];
            bool p = kin && ro >= 0;
            cp_async8(&s[r * C::kLd + kk], p ? (const void *)(G + ro + ko) : (const void *)G, p);
        }
    }
}

template<class C>
__device__ __forceinline__ void load_stage(double *sA, double *sB, const int64_t *rowA,
    const int64_t *rowB, const double *__restrict__ A, const double *__restrict__ B,
    const DTask &t, int k0) {
    load_operand<C, C::BM>(sA, rowA, A, k0, t.K, t.nk, t.kext, t.ka_str, t.vec_a != 0);
    load_operand<C, C::BN>(sB, rowB, B, k0, t.K, t.nk, t.kext, t.kb_str, t.vec_b != 0);
}

// SCATTER: the epilogue writes each C block's tile to the destinations
// dests[drange[cblk].x .. drange[cblk].y) instead of the block itself --
// blocks of another tensor, each through its own index mapping and scale
// (the terms of a symmetrizer over the contraction) -- by atomic adds into
// a zeroed result.
template<class C, bool SCATTER>
__global__ void __launch_bounds__(C::kThreads, C::MINB)
contract_fp64_kernel(const DTask *__restrict__ tasks, const DCBlock *__restrict__ cblks,
                     const DItem *__restrict__ items, int32_t nitems, int32_t *counter,
                     const double *__restrict__ A, const double *__restrict__ B,
                     double *__restrict__ Cp, double *__restrict__ ws, int32_t add,
                     const int2 *__restrict__ drange, const DCBlock *__restrict__ dests) {
    extern __shared__ __align__(16) double smem[];
    double *sA = smem;
    double *sB = smem + C::STAGES * C::kStageA;
    int64_t *rowA = reinterpret_cast<int64_t *>(sB + C::STAGES * C::kStageB);
    int64_t *rowB = rowA + C::BM;
    __shared__ int32_t s_item;
    __shared__ __align__(16) DTask s_task;

    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t4 = lane & 3;
    const int wm = warp / C::kWarpsN, wn = warp % C::kWarpsN;

    while (true) {
        if (tid == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int it = s_item;
        __syncthreads();
        if (it >= nitems) break;
        const DItem item = items[it];
        const DCBlock &cb = cblks[item.cblk];
        const int M = cb.M, N = cb.N;

        // lane fragment q of tile (i, j): row i * kFragRows + g + 8 (q >> 1),
        // column j * 8 + 2 t4 + (q & 1) of the warp tile
        double acc[C::kMT][C::kNT][C::kQ];
#pragma unroll
        for (int i = 0; i < C::kMT; i++)
#pragma unroll
            for (int j = 0; j < C::kNT; j++)
#pragma unroll
                for (int q = 0; q < C::kQ; q++) acc[i][j][q] = 0.0;

        int kt_base = 0;                       // k tiles of the tasks before ti
        for (int ti = cb.t_begin; ti < cb.t_end && kt_base < item.kt1; ti++) {
            // this item's k tiles of the task (a k chunk may cover part of it)
            const int nkt_task = (tasks[ti].K + C::BK - 1) / C::BK;
            const int kt_lo = max(item.kt0 - kt_base, 0);
            const int kt_hi = min(item.kt1 - kt_base, nkt_task);
            kt_base += nkt_task;
            if (kt_lo >= kt_hi) continue;
            static_assert(sizeof(DTask) % 8 == 0, "task copy granularity");
            if (tid < (int)(sizeof(DTask) / 8))
                reinterpret_cast<int64_t *>(&s_task)[tid] =
                    reinterpret_cast<const int64_t *>(&tasks[ti])[tid];
            __syncthreads();
            const DTask &t = s_task;
            for (int r = tid; r < C::BM; r += C::kThreads) {
                int m = item.m0 + r;
                rowA[r] = m < M ? t.a_off + mixed_offset(m, t.nm, t.mext, t.ma_str) : -1;
            }
            for (int r = tid; r < C::BN; r += C::kThreads) {
                int n = item.n0 + r;
                rowB[r] = n < N ? t.b_off + mixed_offset(n, t.nn, t.next, t.nb_str) : -1;
            }
            __syncthreads();
            const double coef = t.coeff;
            const bool scale_b = coef != 1.0;
            const int nkt = kt_hi - kt_lo;          // k tiles kt_lo + kt, kt = 0 .. nkt-1

#pragma unroll
            for (int s = 0; s < C::STAGES - 1; s++) {
                if (s < nkt)
                    load_stage<C>(sA + s * C::kStageA, sB + s * C::kStageB, rowA, rowB, A, B, t,
                                  (kt_lo + s) * C::BK);
                cp_async_commit();
            }
            for (int kt = 0; kt < nkt; kt++) {
                cp_async_wait<C::STAGES - 2>();
                __syncthreads();
                {
                    int nk = kt + C::STAGES - 1;
                    if (nk < nkt) {
                        int st = nk % C::STAGES;
                        load_stage<C>(sA + st * C::kStageA, sB + st * C::kStageB, rowA, rowB, A, B, t,
                                      (kt_lo + nk) * C::BK);
                    }
                    cp_async_commit();
                }
                const int st = kt % C::STAGES;
                if constexpr (C::MMA == kMma8x8x4) {
                    // one double per fragment: A[g][k], B[n = g][k], k = ks + t4
                    const double *tA = sA + st * C::kStageA + (wm * C::WM + g) * C::kLd + t4;
                    const double *tB = sB + st * C::kStageB + (wn * C::WN + g) * C::kLd + t4;
                    double af[2][C::kMT], bf[2][C::kNT];
                    auto load8 = [&](int buf, int ks) {
#pragma unroll
                        for (int i = 0; i < C::kMT; i++) af[buf][i] = tA[(i * 8) * C::kLd + ks];
#pragma unroll
                        for (int j = 0; j < C::kNT; j++) bf[buf][j] = tB[(j * 8) * C::kLd + ks];
                    };
                    load8(0, 0);
#pragma unroll
                    for (int ks = 0; ks < C::BK; ks += 4) {
                        const int cur = (ks / 4) & 1;
                        if (ks + 4 < C::BK) load8(cur ^ 1, ks + 4);
                        if (scale_b) {
#pragma unroll
                            for (int j = 0; j < C::kNT; j++) bf[cur][j] *= coef;
                        }
#pragma unroll
                        for (int i = 0; i < C::kMT; i++)
#pragma unroll
                            for (int j = 0; j < C::kNT; j++) dmma_8x8x4(acc[i][j], af[cur][i], bf[cur][j]);
                    }
                } else {
                const double *tA = sA + st * C::kStageA + (wm * C::WM + g) * C::kLd + 2 * t4;
                const double *tB = sB + st * C::kStageB + (wn * C::WN + g) * C::kLd + 2 * t4;
                double af[2][C::kMT][4], bf[2][C::kNT][2];
                auto load_frags = [&](int buf, int ks) {
#pragma unroll
                    for (int i = 0; i < C::kMT; i++) {
                        double2 lo = *reinterpret_cast<const double2 *>(tA + (i * 16) * C::kLd + ks);
                        double2 hi = *reinterpret_cast<const double2 *>(tA + (i * 16 + 8) * C::kLd + ks);
                        af[buf][i][0] = lo.x; af[buf][i][2] = lo.y; af[buf][i][1] = hi.x; af[buf][i][3] = hi.y;
                    }
#pragma unroll
                    for (int j = 0; j < C::kNT; j++) {
                        double2 v = *reinterpret_cast<const double2 *>(tB + (j * 8) * C::kLd + ks);
                        bf[buf][j][0] = v.x;
                        bf[buf][j][1] = v.y;
                    }
                };
                if constexpr (C::K16) {
                    // both fragment buffers hold one k16 step
#pragma unroll
                    for (int ks = 0; ks < C::BK; ks += 16) {
                        load_frags(0, ks);
                        load_frags(1, ks + 8);
                        if (scale_b) {
#pragma unroll
                            for (int j = 0; j < C::kNT; j++)
#pragma unroll
                                for (int h = 0; h < 2; h++) { bf[h][j][0] *= coef; bf[h][j][1] *= coef; }
                        }
#pragma unroll
                        for (int i = 0; i < C::kMT; i++)
#pragma unroll
                            for (int j = 0; j < C::kNT; j++)
                                dmma_16x8x16(acc[i][j], af[0][i], af[1][i], bf[0][j], bf[1][j]);
                    }
                } else {
                    load_frags(0, 0);
#pragma unroll
                    for (int ks = 0; ks < C::BK; ks += 8) {
                        const int cur = (ks / 8) & 1;
                        if (ks + 8 < C::BK) load_frags(cur ^ 1, ks + 8);
                        if (scale_b) {
#pragma unroll
                            for (int j = 0; j < C::kNT; j++) { bf[cur][j][0] *= coef; bf[cur][j][1] *= coef; }
                        }
#pragma unroll
                        for (int i = 0; i < C::kMT; i++)
#pragma unroll
                            for (int j = 0; j < C::kNT; j++) dmma_16x8x8(acc[i][j], af[cur][i], bf[cur][j]);
                    }
                }
                }
            }
            cp_async_wait<0>();
            __syncthreads();
        }

        if (item.slot >= 0) {
            // k chunk: the unscaled partial tile, dense BM x BN, to its slot
            double *P = ws + (int64_t)item.slot * (C::BM * C::BN);
#pragma unroll
            for (int i = 0; i < C::kMT; i++)
#pragma unroll
                for (int j = 0; j < C::kNT; j++)
#pragma unroll
                    for (int h = 0; h < C::kQ / 2; h++) {
                        const int r = wm * C::WM + i * C::kFragRows + g + 8 * h;
                        const int cc = wn * C::WN + j * 8 + 2 * t4;
                        *reinterpret_cast<double2 *>(P + r * C::BN + cc) =
                            make_double2(acc[i][j][2 * h], acc[i][j][2 * h + 1]);
                    }
            continue;
        }

        if constexpr (SCATTER) {
            const int2 dr = drange[item.cblk];
            for (int d = dr.x; d < dr.y; d++) {
                const DCBlock &db = dests[d];
                int64_t dm[C::kMT][C::kQ / 2];
                int64_t dn[C::kNT][2];
#pragma unroll
                for (int i = 0; i < C::kMT; i++)
#pragma unroll
                    for (int h = 0; h < C::kQ / 2; h++) {
                        int m = item.m0 + wm * C::WM + i * C::kFragRows + g + 8 * h;
                        dm[i][h] = m < M ? mixed_offset(m, db.nm, db.mext, db.mc_str) : -1;
                    }
#pragma unroll
                for (int j = 0; j < C::kNT; j++)
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        int n = item.n0 + wn * C::WN + j * 8 + 2 * t4 + h;
                        dn[j][h] = n < N ? mixed_offset(n, db.nn, db.next, db.nc_str) : -1;
                    }
                double *Db = Cp + db.c_off;
#pragma unroll
                for (int i = 0; i < C::kMT; i++)
#pragma unroll
                    for (int j = 0; j < C::kNT; j++)
#pragma unroll
                        for (int q = 0; q < C::kQ; q++) {
                            int64_t om = dm[i][q >> 1], on = dn[j][q & 1];
                            if (om < 0 || on < 0) continue;
                            atomicAdd(Db + om + on, db.scale * acc[i][j][q]);
                        }
            }
            continue;
        }

        // Epilogue: scaled store (assign) or scaled accumulate (add) into the
        // canonical C block through its own index mapping.
        const double scale = cb.scale;
        int64_t coff_m[C::kMT][C::kQ / 2];
        int64_t coff_n[C::kNT][2];
#pragma unroll
        for (int i = 0; i < C::kMT; i++)
#pragma unroll
            for (int h = 0; h < C::kQ / 2; h++) {
                int m = item.m0 + wm * C::WM + i * C::kFragRows + g + 8 * h;
                coff_m[i][h] = m < M ? mixed_offset(m, cb.nm, cb.mext, cb.mc_str) : -1;
            }
#pragma unroll
        for (int j = 0; j < C::kNT; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                int n = item.n0 + wn * C::WN + j * 8 + 2 * t4 + h;
                coff_n[j][h] = n < N ? mixed_offset(n, cb.nn, cb.next, cb.nc_str) : -1;
            }
        double *Cb = Cp + cb.c_off;
#pragma unroll
        for (int i = 0; i < C::kMT; i++)
#pragma unroll
            for (int j = 0; j < C::kNT; j++)
#pragma unroll
                for (int q = 0; q < C::kQ; q++) {
                    int64_t om = coff_m[i][q >> 1], on = coff_n[j][q & 1];
                    if (om < 0 || on < 0) continue;
                    double v = scale * acc[i][j][q];
                    if (add) Cb[om + on] += v;
                    else Cb[om + on] = v;
                }
    }
}

// Split tiles: element e of tile x sums its nparts partials in chunk order
// (fixed order: the result does not depend on which CTA ran which chunk).
__global__ void __launch_bounds__(256)
split_reduce_kernel(const DSplit *__restrict__ splits, int32_t nsplits, const DCBlock *__restrict__ cblks,
                    const double *__restrict__ ws, int32_t bm, int32_t bn, double *__restrict__ Cp,
                    int32_t add) {
    const int64_t tile = (int64_t)bm * bn;
    const int64_t total = (int64_t)nsplits * tile;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t x = (int32_t)(e / tile);
        const int32_t r = (int32_t)((e - (int64_t)x * tile) / bn);
        const int32_t cc = (int32_t)(e - (int64_t)x * tile - (int64_t)r * bn);
        const DSplit sp = splits[x];
        const DCBlock &cb = cblks[sp.cblk];
        const int m = sp.m0 + r, n = sp.n0 + cc;
        if (m >= cb.M || n >= cb.N) continue;
        const double *p = ws + (int64_t)sp.slot0 * tile + (int64_t)r * bn + cc;
        double v = 0.0;
        for (int q = 0; q < sp.nparts; q++) v += p[(int64_t)q * tile];
        v *= cb.scale;
        double *dst = Cp + cb.c_off + mixed_offset(m, cb.nm, cb.mext, cb.mc_str) +
                      mixed_offset(n, cb.nn, cb.next, cb.nc_str);
        if (add) *dst += v;
        else *dst = v;
    }
}

template<class C, bool SCATTER>
cudaError_t launch_cfg_s(const DTask *tasks, const DCBlock *cblks, const DItem *items,
                         int32_t nitems, int32_t *counter, const double *a, const double *b,
                         double *c, double *ws, int32_t add, const int2 *drange, const DCBlock *dests,
                         cudaStream_t s) {
    static int configured_dev = -1;
    cudaError_t e;
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    if (configured_dev != dev) {
        e = cudaFuncSetAttribute(contract_fp64_kernel<C, SCATTER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)C::kSmem);
        if (e != cudaSuccess) return e;
        configured_dev = dev;
    }
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    int grid = nitems < nsm * C::MINB ? nitems : nsm * C::MINB;       // persistent: resident CTAs
    if (grid < 1) return cudaSuccess;
    e = cudaMemsetAsync(counter, 0, sizeof(int32_t), s);
    if (e != cudaSuccess) return e;
    contract_fp64_kernel<C, SCATTER><<<grid, C::kThreads, C::kSmem, s>>>(tasks, cblks, items, nitems, counter,
                                                                        a, b, c, ws, add, drange, dests);
    return cudaGetLastError();
}

template<class C>
cudaError_t launch_cfg(const DTask *tasks, const DCBlock *cblks, const DItem *items,
                       int32_t nitems, int32_t *counter, const double *a, const double *b,
                       double *c, double *ws, int32_t add, const int2 *drange, const DCBlock *dests,
                       cudaStream_t s) {
    if (dests)
        return launch_cfg_s<C, true>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    return launch_cfg_s<C, false>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, nullptr, nullptr, s);
}

// Tile configurations (BM, BN, BK, warp tile M, warp tile N, stages).
using Cfg0 = TileCfg<128, 128, 16, 64, 32, 4>;
using Cfg1 = TileCfg<64, 64, 32, 32, 32, 3>;
using Cfg2 = TileCfg<64, 128, 32, 32, 32, 3>;
using Cfg3 = TileCfg<32, 32, 32, 16, 16, 3>;
using Cfg4 = TileCfg<80, 128, 32, 80, 16, 3>;
using Cfg5 = TileCfg<96, 128, 32, 96, 16, 3>;
using Cfg6 = TileCfg<48, 128, 32, 48, 16, 3>;
using Cfg7 = TileCfg<112, 128, 16, 112, 16, 4>;
// short shapes for C blocks of 16 or 32 rows (e.g. an occupied pair block
// of 4 x 4 orbitals): wide in N so that each A row slab is reused 128 times
using Cfg8 = TileCfg<16, 128, 32, 16, 16, 3>;
using Cfg9 = TileCfg<32, 128, 32, 32, 16, 3>;
// 80-row shapes with twelve warps (three per scheduler, 168 registers)
using Cfg10 = TileCfg<80, 192, 16, 80, 16, 4>;
using Cfg11 = TileCfg<80, 192, 32, 80, 16, 2>;
// m16n8k16 DMMA forms of shapes 11 and 4, and a squarer warp tile (48 x 32:
// 12 DMMAs per 10 fragment loads instead of 10 per 12)
using Cfg12 = TileCfg<80, 192, 32, 80, 16, 2, true>;
using Cfg13 = TileCfg<80, 128, 32, 80, 16, 3, true>;
using Cfg14 = TileCfg<96, 128, 32, 48, 32, 3>;
// m8n8k4 DMMA (one double per fragment): 40 x 32 warp tiles (80-row C
// tiles), and a 64 x 128 tile of 32 x 64 warp tiles, two CTAs per SM
using Cfg15 = TileCfg<80, 128, 32, 40, 32, 3, kMma8x8x4>;
using Cfg16 = TileCfg<80, 192, 32, 40, 32, 2, kMma8x8x4>;
using Cfg17 = TileCfg<64, 128, 16, 32, 64, 3, kMma8x8x4, 2>;
// more m8n8k4 shapes with two CTAs per SM: 80-row tiles of 40 x 64 and
// 40 x 32 warp tiles, BK 32 with two stages, and 128 x 64
using Cfg18 = TileCfg<80, 128, 16, 40, 64, 3, kMma8x8x4, 2>;
using Cfg19 = TileCfg<80, 128, 16, 40, 32, 3, kMma8x8x4, 2>;
using Cfg20 = TileCfg<64, 128, 32, 32, 64, 2, kMma8x8x4, 2>;
using Cfg21 = TileCfg<128, 64, 16, 64, 32, 3, kMma8x8x4, 2>;

}  // namespace

int tile_cfg_count() { return 22; }
int tile_cfg_bm(int cfg) {
    const int v[] = {Cfg0::BM, Cfg1::BM, Cfg2::BM, Cfg3::BM, Cfg4::BM, Cfg5::BM, Cfg6::BM, Cfg7::BM, Cfg8::BM, Cfg9::BM, Cfg10::BM, Cfg11::BM, Cfg12::BM, Cfg13::BM, Cfg14::BM, Cfg15::BM, Cfg16::BM, Cfg17::BM, Cfg18::BM, Cfg19::BM, Cfg20::BM, Cfg21::BM};
    return v[cfg];
}
int tile_cfg_bk(int cfg) {
    const int v[] = {Cfg0::BK, Cfg1::BK, Cfg2::BK, Cfg3::BK, Cfg4::BK, Cfg5::BK, Cfg6::BK, Cfg7::BK, Cfg8::BK, Cfg9::BK, Cfg10::BK, Cfg11::BK, Cfg12::BK, Cfg13::BK, Cfg14::BK, Cfg15::BK, Cfg16::BK, Cfg17::BK, Cfg18::BK, Cfg19::BK, Cfg20::BK, Cfg21::BK};
    return v[cfg];
}
int tile_cfg_bn(int cfg) {
    const int v[] = {Cfg0::BN, Cfg1::BN, Cfg2::BN, Cfg3::BN, Cfg4::BN, Cfg5::BN, Cfg6::BN, Cfg7::BN, Cfg8::BN, Cfg9::BN, Cfg10::BN, Cfg11::BN, Cfg12::BN, Cfg13::BN, Cfg14::BN, Cfg15::BN, Cfg16::BN, Cfg17::BN, Cfg18::BN, Cfg19::BN, Cfg20::BN, Cfg21::BN};
    return v[cfg];
}

cudaError_t launch_split_reduce(const DSplit *splits, int32_t nsplits, const DCBlock *cblks,
    const double *ws, int32_t bm, int32_t bn, double *c, int32_t add, cudaStream_t s) {
    if (nsplits <= 0) return cudaSuccess;
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int64_t total = (int64_t)nsplits * bm * bn;
    const int64_t want = (total + 255) / 256;
    // one wave of resident CTAs (a partial last wave would set the time)
    static const int per_sm = [] {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, split_reduce_kernel, 256, 0) != cudaSuccess || n < 1) n = 1;
        return n;
    }();
    const int grid = (int)(want < (int64_t)per_sm * nsm ? want : (int64_t)per_sm * nsm);
    split_reduce_kernel<<<grid, 256, 0, s>>>(splits, nsplits, cblks, ws, bm, bn, c, add);
    return cudaGetLastError();
}

cudaError_t launch_contract_fp64(const DTask *tasks, const DCBlock *cblks,
    const DItem *items, int32_t nitems, int32_t *counter, const double *a,
    const double *b, double *c, double *ws, int32_t add, int32_t tile_cfg, cudaStream_t s,
    const int2 *drange, const DCBlock *dests) {
    switch (tile_cfg) {
    case 0: return launch_cfg<Cfg0>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    case 1: return launch_cfg<Cfg1>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    case 2: return launch_cfg<Cfg2>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    case 3: return launch_cfg<Cfg3>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    case 4: return launch_cfg<Cfg4>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    case 5: return launch_cfg<Cfg5>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    case 6: return launch_cfg<Cfg6>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    case 7: return launch_cfg<Cfg7>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    case 8: return launch_cfg<Cfg8>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    case 9: return launch_cfg<Cfg9>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    case 10: return launch_cfg<Cfg10>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    case 11: return launch_cfg<Cfg11>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    case 12: return launch_cfg<Cfg12>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    case 13: return launch_cfg<Cfg13>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    case 14: return launch_cfg<Cfg14>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    case 15: return launch_cfg<Cfg15>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    case 16: return launch_cfg<Cfg16>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    case 17: return launch_cfg<Cfg17>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    case 18: return launch_cfg<Cfg18>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    case 19: return launch_cfg<Cfg19>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    case 20: return launch_cfg<Cfg20>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    default: return launch_cfg<Cfg21>(tasks, cblks, items, nitems, counter, a, b, c, ws, add, drange, dests, s);
    }
}

}  // namespace ltg
