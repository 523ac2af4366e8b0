// Split-precision ("Ozaki scheme") block-pair contraction on the B200 5th
// generation tensor cores (tcgen05.mma, accumulators in tensor memory).
//
// Same schedule and task list as the plain FP64 path (one work item per
// (C block, 128-row, 64-column) tile, all coalesced pairs of the C block
// accumulated before the single FP64 write), but the products run on
// integer-valued low-precision slices:
//
//  1. split (oz_split_kernel): every matricised operand row r of a block is
//     scaled by its own power of two 2^-e_r (e_r: exponent of the row's
//     largest magnitude) and cut into S slices of integers by round-to-nearest,
//       x = 2^(e_r - b0) * sum_s sigma_s * 2^(-b*s),  |sigma_s| <= 2^(b0) or 2^(b-1),
//     exactly, up to the dropped tail (Ozaki, Ogita, Oishi, Rump 2012; the
//     per-row power-of-two scaling of Mukunoki et al. 2020).  The permutation
//     of the block pair is applied here, so the slices are GEMM-ready.
//  2. slice products (oz_gemm_kernel): the products sigma_sa x sigma_sb with
//     sa + sb = l (a "level") share one scale, so each level accumulates in its
//     own TMEM accumulator.  INT8 slices accumulate exactly in INT32; BF16 and
//     FP8 E4M3 slices accumulate in FP32, exact while every partial sum stays
//     below 2^24, which the host guarantees by draining every chunk_kb k blocks.
//  3. recombination: after each pair (or chunk) the epilogue warps read the
//     level accumulators from TMEM and add
//       coeff * 2^(e_r + e_c - 2 b0) * sum_l 2^(-b l) * acc_l
//     into FP64 registers; the C tile is written once, in FP64.
// Only levels l <= S-1 are formed: S(S+1)/2 slice products per k step.
//
// Warp roles (192 threads): warps 0-3 epilogue (TMEM lanes 0-127, one C row
// per thread), warp 4 bulk-copy producer, warp 5 MMA issuer.  Operand tiles
// are stored in global memory as the exact shared-memory images the MMA reads
// (K-major core matrices, no swizzle), so each one moves with a single 1-D
// cp.async.bulk copy completing on the stage's mbarrier (no tensor maps, no
// multicast); one MMA k step per pipeline stage, so even 8 slices leave room
// for 4 stages.
// Every mbarrier wait is bounded in time and reports through *err.
#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include "ltg_device.cuh"

namespace ltg {

// k elements per 32-byte k block: 32 for 8-bit slices, 16 for BF16.
void oz_kind_params(int kind, int *beta0, int *beta, int *esz, int *kbe, int64_t *maxprod) {
    switch (kind) {
    case kOzInt8: *beta0 = 6; *beta = 7; *esz = 1; *kbe = 32; *maxprod = 64 * 64; break;
    case kOzBf16: *beta0 = 6; *beta = 7; *esz = 2; *kbe = 16; *maxprod = 64 * 64; break;
    default:      *beta0 = 4; *beta = 5; *esz = 1; *kbe = 32; *maxprod = 16 * 16; break;
    }
}

namespace {

constexpr int kBM = 128;              // C rows per tile (TMEM lanes)
constexpr int kBN = 64;               // C columns per tile (TMEM columns per level)
constexpr int kRowBytes = 32;         // k-block row length in shared memory (one MMA k step)
constexpr int kATile = kBM * kRowBytes;   // 4 KB per A slice per stage
constexpr int kBTile = kBN * kRowBytes;   // 2 KB per B slice per stage
constexpr int kThreads = 192;
constexpr int kMaxStages = 8;
constexpr uint64_t kWaitNs = 2000000000ull;   // 2 s: the drain waits after an abort

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

// ---------------------------------------------------------------- split

// Four consecutive slice values packed for one store.
template<int KIND> struct Pack4;
template<> struct Pack4<kOzInt8> {
    typedef uint32_t T;
    __device__ static T pack(const double *v) {
        return (uint32_t)(uint8_t)(int8_t)(int)v[0] | ((uint32_t)(uint8_t)(int8_t)(int)v[1] << 8) |
               ((uint32_t)(uint8_t)(int8_t)(int)v[2] << 16) | ((uint32_t)(uint8_t)(int8_t)(int)v[3] << 24);
    }
};
template<> struct Pack4<kOzE4m3> {
    typedef uint32_t T;
    __device__ static T pack(const double *v) {
        uint32_t r = 0;
        for (int i = 0; i < 4; i++) {
            __nv_fp8_e4m3 q((float)v[i]);
            r |= (uint32_t)q.__x << (8 * i);
        }
        return r;
    }
};
template<> struct Pack4<kOzBf16> {
    typedef uint2 T;
    __device__ static T pack(const double *v) {
        __nv_bfloat16 b[4];
        for (int i = 0; i < 4; i++) b[i] = __float2bfloat16_rn((float)v[i]);
        uint2 r;
        r.x = (uint32_t)__bfloat16_as_ushort(b[0]) | ((uint32_t)__bfloat16_as_ushort(b[1]) << 16);
        r.y = (uint32_t)__bfloat16_as_ushort(b[2]) | ((uint32_t)__bfloat16_as_ushort(b[3]) << 16);
        return r;
    }
};

// Byte offset of (row r, byte kb_byte of k block kb, slice s) in the tile
// images of a panel.  Panels are stored as the exact shared-memory images
// the MMA reads: per (row tile, k block, slice) one TR x 32-byte tile,
// K-major without swizzle (8-row x 16-byte core matrices, the two 16-byte k
// halves 128 bytes apart, 8-row groups 256 bytes apart), so one pipeline
// stage is a single contiguous bulk copy per operand.
__device__ __forceinline__ int64_t tile_image_offset(int r, int TR, int nkb, int kb, int s, int S,
                                                     int kb_byte) {
    const int tile = r / TR, rr = r % TR;
    return ((int64_t)(tile * nkb + kb) * S + s) * (TR * 32) + (rr >> 3) * 256 + (kb_byte >> 4) * 128 +
           (rr & 7) * 16 + (kb_byte & 15);
}

// 32 panel rows per CTA, 8 threads per row, 4 consecutive k per thread; two
// passes over each row (largest magnitude, then the slices).  Contiguous
// rows (one k sub-dimension of stride 1) skip the mixed-radix arithmetic.
template<int KIND>
__global__ void __launch_bounds__(256)
oz_split_kernel(const DPanel *__restrict__ panels, int32_t npanels,
                const double *__restrict__ A, const double *__restrict__ B,
                uint8_t *__restrict__ slices, int32_t *__restrict__ exps, int32_t S,
                int32_t beta0, int32_t beta) {
    typedef typename Pack4<KIND>::T PT;
    constexpr int kEsz = KIND == kOzBf16 ? 2 : 1;
    constexpr int kKbe = 32 / kEsz;                  // elements per 32-byte k block
    const int lr = threadIdx.x >> 3;                 // row within the CTA's 32 rows
    const int c = threadIdx.x & 7;                   // 4-element chunk of a 32-element step
    for (int p = blockIdx.y; p < npanels; p += gridDim.y) {
        const DPanel &P = panels[p];
        const double *src = P.src ? B : A;
        uint8_t *base = slices + P.slice_off;
        const int TR = P.src ? 64 : 128;             // rows per tile image (MMA N or M)
        const int nkb = P.K_pad / kKbe;
        const bool contig = P.nk == 1 && P.kstr[0] == 1;
        for (int r0 = blockIdx.x * 32; r0 < P.rows_pad; r0 += gridDim.x * 32) {
            const int r = r0 + lr;
            const bool valid = r < P.rows;
            const double *row = src + (valid ? P.src_off + mixed_offset(r, P.nr, P.rext, P.rstr) : 0);
            double mx = 0.0;
            if (valid)
                for (int k0 = 4 * c; k0 < P.K; k0 += 32)
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        const int k = k0 + j;
                        if (k < P.K) mx = fmax(mx, fabs(row[contig ? k : mixed_offset(k, P.nk, P.kext, P.kstr)]));
                    }
            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 2));
            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 4));
            int e = 0;
            if (mx > 0.0) frexp(mx, &e);            // mx = f * 2^e, f in [0.5, 1)
            if (c == 0) exps[P.exp_off + r] = e;
            const double up = ldexp(1.0, beta);
            for (int k0 = 4 * c; k0 < P.K_pad; k0 += 32) {
                double t[4], sg[4];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int k = k0 + j;
                    const double x = (valid && k < P.K) ? row[contig ? k : mixed_offset(k, P.nk, P.kext, P.kstr)] : 0.0;
                    t[j] = ldexp(x, beta0 - e);     // |t| < 2^beta0, exact
                }
                const int kb = k0 / kKbe, kb_byte = (k0 % kKbe) * kEsz;
                for (int s = 0; s < S; s++) {
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        sg[j] = rint(t[j]);
                        t[j] = (t[j] - sg[j]) * up;   // exact (Sterbenz), power-of-two scale
                    }
                    *reinterpret_cast<PT *>(base + tile_image_offset(r, TR, nkb, kb, s, S, kb_byte)) =
                        Pack4<KIND>::pack(sg);
                }
            }
        }
    }
}

// ---------------------------------------------------------------- tcgen05 helpers

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("{ .reg .b64 st; mbarrier.arrive.shared::cta.b64 st, [%0]; }" :: "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("{ .reg .b64 st; mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1; }"
                 :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for the phase with the given parity to complete, for at most
// limit_ns of wall time (try_wait itself may suspend the thread, so the bound
// is on time, not on iterations); false on timeout or when another role
// aborted.  limit_ns == 0 tests the phase once and does not wait.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *abort,
                                          uint64_t limit_ns) {
    const uint32_t a = smem_u32(bar);
    if (limit_ns == 0) {                 // no time at all: one non-blocking test
        uint32_t done;
        asm volatile("{ .reg .pred p; mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                     : "=r"(done) : "r"(a), "r"(parity) : "memory");
        return done != 0;
    }
    uint64_t t0 = 0;
    for (uint32_t i = 0;; i++) {
        uint32_t done;
        asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                     : "=r"(done) : "r"(a), "r"(parity) : "memory");
        if (done) return true;
        if ((i & 63) == 63) {
            if (*abort) return false;
            const uint64_t t = global_ns();
            if (t0 == 0) t0 = t;
            else if (t - t0 > limit_ns) return false;
        }
    }
}

// One contiguous global -> shared bulk copy (16-byte aligned, size a
// multiple of 16), completing on the stage's mbarrier.  No multicast.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        :: "r"(dst), "l"(src), "r"(bytes), "r"(bar) : "memory");
}

// K-major shared-memory matrix descriptor without swizzle: 8-row x 16-byte
// core matrices, the two k halves 128 bytes apart (leading byte offset),
// 8-row groups 256 bytes apart (stride byte offset).
__device__ __forceinline__ uint64_t smem_desc_kmajor(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);          // start address
    d |= (uint64_t)(128 >> 4) << 16;                  // leading byte offset
    d |= (uint64_t)(256 >> 4) << 32;                  // stride byte offset
    d |= (uint64_t)1 << 46;                           // descriptor version (sm_100)
    return d;                                         // layout type 0: no swizzle
}

template<int KIND>
__device__ __forceinline__ uint32_t instr_desc() {
    // D format: S32 for int8, F32 otherwise; A/B formats; K-major A and B;
    // N = 64, M = 128.
    uint32_t c_fmt = KIND == kOzInt8 ? 2u : 1u;
    uint32_t ab_fmt = KIND == kOzInt8 ? 1u : (KIND == kOzBf16 ? 1u : 0u);
    return (c_fmt << 4) | (ab_fmt << 7) | (ab_fmt << 10) | ((uint32_t)(kBN >> 3) << 17) |
           ((uint32_t)(kBM >> 4) << 24);
}

template<int KIND>
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                     uint32_t accumulate) {
    if (KIND == kOzInt8) {
        asm volatile("{ .reg .pred p; setp.ne.b32 p, %4, 0;\n"
                     "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p; }"
                     :: "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate) : "memory");
    } else if (KIND == kOzBf16) {
        asm volatile("{ .reg .pred p; setp.ne.b32 p, %4, 0;\n"
                     "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p; }"
                     :: "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate) : "memory");
    } else {
        asm volatile("{ .reg .pred p; setp.ne.b32 p, %4, 0;\n"
                     "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p; }"
                     :: "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate) : "memory");
    }
}

// Same product with the A operand read from tensor memory (a_tmem).
template<int KIND>
__device__ __forceinline__ void umma_ts(uint32_t tmem_d, uint32_t a_tmem, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
    if (KIND == kOzInt8) {
        asm volatile("{ .reg .pred p; setp.ne.b32 p, %4, 0;\n"
                     "tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, p; }"
                     :: "r"(tmem_d), "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accumulate) : "memory");
    } else if (KIND == kOzBf16) {
        asm volatile("{ .reg .pred p; setp.ne.b32 p, %4, 0;\n"
                     "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p; }"
                     :: "r"(tmem_d), "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accumulate) : "memory");
    } else {
        asm volatile("{ .reg .pred p; setp.ne.b32 p, %4, 0;\n"
                     "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], [%1], %2, %3, p; }"
                     :: "r"(tmem_d), "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accumulate) : "memory");
    }
}

// Shared -> tensor memory copy of one 128-row x 32-byte operand tile (row r
// to TMEM lane r, 8 columns).  Executes in issue order with the MMAs of the
// same thread, so a single A buffer can be refilled every k step.
__device__ __forceinline__ void tmem_cp_128x256b(uint32_t taddr, uint64_t sdesc) {
    asm volatile("tcgen05.cp.cta_group::1.128x256b [%0], %1;" :: "r"(taddr), "l"(sdesc) : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t *v) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                   "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr) : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// ---------------------------------------------------------------- slice products

// SCATTER: each finished tile row goes, by atomic adds into a zeroed
// result, to the destinations dests[drange[cblk]] of its C block (blocks of
// another tensor with their own index mappings and scales: the terms of a
// symmetrizer over the contraction) instead of the C block itself.
template<int KIND, int S, bool SCATTER = false>
__global__ void __launch_bounds__(kThreads, 1)
oz_gemm_kernel(const DPanel *__restrict__ panels, const uint8_t *__restrict__ slices,
               const DOzTask *__restrict__ tasks, const DCBlock *__restrict__ cblks,
               const DItem *__restrict__ items, int32_t nitems, const int32_t *__restrict__ exps,
               double *__restrict__ Cp, int32_t add, int32_t stages, int32_t chunk_kb,
               int32_t beta0, int32_t beta, int32_t kbe, int32_t *err, uint64_t wait_ns,
               const int2 *__restrict__ drange = nullptr, const DCBlock *__restrict__ dests = nullptr) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // 1024-byte aligned stage buffers: [stage][A slices | B slices]
    uint8_t *smem = reinterpret_cast<uint8_t *>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    constexpr int kStageBytes = S * (kATile + kBTile);
    // A operand from tensor memory (tcgen05.cp of the A slices once per k
    // step, products reading only B from shared memory) is supported when the
    // accumulators leave room for it, but measured slower than reading both
    // operands from shared memory on the ladder workloads (35.1 vs 39.4
    // effective TFLOP/s at S = 7), so it is off.
    constexpr bool kATmem = false && (S * kBN + S * 8 <= 512);
    constexpr int kACol = S * kBN;
    __shared__ __align__(8) uint64_t full_bar[kMaxStages], empty_bar[kMaxStages], accf_bar, acce_bar, drain_bar;
    __shared__ uint32_t tmem_base_s;
    __shared__ volatile int abort_s;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int i = 0; i < stages; i++) { mbar_init(&full_bar[i], 1); mbar_init(&empty_bar[i], 1); }
        mbar_init(&accf_bar, 1);
        mbar_init(&acce_bar, 4);
        mbar_init(&drain_bar, 1);
        abort_s = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;"
                     :: "r"(smem_u32(&tmem_base_s)) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_s;
    const uint32_t smem0 = smem_u32(smem);

    if (warp == 4) {
        // ------------------------------------------------ bulk-copy producer (1-D cp.async.bulk)
        if (lane == 0) {
            int st = 0;
            uint32_t ph = 0;
            bool ok = true;
            int armed_parity[kMaxStages];
            for (int i = 0; i < kMaxStages; i++) armed_parity[i] = -1;
            for (int it = blockIdx.x; it < nitems && ok; it += gridDim.x) {
                const DItem item = items[it];
                const DCBlock &cb = cblks[item.cblk];
                for (int ti = cb.t_begin; ti < cb.t_end && ok; ti++) {
                    const DOzTask t = tasks[ti];
                    const int nkb = panels[t.pa].K_pad / kbe;
                    // tile images of this (row tile, k block): all S slices contiguous
                    const uint8_t *ga = slices + panels[t.pa].slice_off + (int64_t)(item.m0 / kBM) * nkb * S * kATile;
                    const uint8_t *gb = slices + panels[t.pb].slice_off + (int64_t)(item.n0 / kBN) * nkb * S * kBTile;
                    for (int kb = 0; kb < nkb; kb++) {
                        if (!mbar_wait(&empty_bar[st], ph ^ 1, &abort_s, wait_ns)) { ok = false; break; }
                        const uint32_t sa = smem0 + st * kStageBytes;
                        const uint32_t sb = sa + S * kATile;
                        const uint32_t fb = smem_u32(&full_bar[st]);
                        mbar_expect_tx(&full_bar[st], (uint32_t)kStageBytes);
                        bulk_load(sa, ga + (int64_t)kb * S * kATile, S * kATile, fb);
                        bulk_load(sb, gb + (int64_t)kb * S * kBTile, S * kBTile, fb);
                        armed_parity[st] = (int)ph;
                        if (++st == stages) { st = 0; ph ^= 1; }
                    }
                }
            }
            if (!ok) {
                abort_s = 1;
                atomicExch(err, 7);
            }
            // let the copies already in flight land before the CTA exits (after
            // an abort the MMA warp no longer consumes them; in a normal run
            // each stage's last phase has completed already)
            volatile int never = 0;
            for (int i = 0; i < stages; i++)
                if (armed_parity[i] >= 0) (void)mbar_wait(&full_bar[i], (uint32_t)armed_parity[i], &never, kWaitNs);
        }
    } else if (warp == 5) {
        // ------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t idesc = instr_desc<KIND>();
            int st = 0;
            uint32_t ph = 0, accph = 0;
            int ndrain = 0;
            bool ok = true;
            for (int it = blockIdx.x; it < nitems && ok; it += gridDim.x) {
                const DItem item = items[it];
                const DCBlock &cb = cblks[item.cblk];
                for (int ti = cb.t_begin; ti < cb.t_end && ok; ti++) {
                    const int nkb = panels[tasks[ti].pa].K_pad / kbe;
                    for (int kb0 = 0; kb0 < nkb && ok; kb0 += chunk_kb) {
                        // the accumulators are free once the previous drain was read
                        if (ndrain > 0) {
                            if (!mbar_wait(&acce_bar, accph, &abort_s, wait_ns)) { ok = false; break; }
                            accph ^= 1;
                        }
                        tc_fence_after();
                        const int kb1 = min(nkb, kb0 + chunk_kb);
                        for (int kb = kb0; kb < kb1; kb++) {
                            if (!mbar_wait(&full_bar[st], ph, &abort_s, wait_ns)) { ok = false; break; }
                            tc_fence_after();
                            const uint32_t a0 = smem0 + st * kStageBytes;
                            const uint32_t b0 = a0 + S * kATile;
                            const uint64_t da = smem_desc_kmajor(a0), db = smem_desc_kmajor(b0);
                            const uint32_t first = kb == kb0 ? 0u : 1u;
                            if (kATmem) {
                                // A slices into tensor memory once per k step; the
                                // products then read only B from shared memory.
#pragma unroll
                                for (int sa = 0; sa < S; sa++)
                                    tmem_cp_128x256b(tmem + (uint32_t)(kACol + sa * 8),
                                                     da + (uint64_t)((sa * kATile) >> 4));
                            }
#pragma unroll
                            for (int l = 0; l < S; l++) {
#pragma unroll
                                for (int sa = 0; sa <= l; sa++) {
                                    const int sb = l - sa;
                                    // descriptor start addresses advance in 16-byte units
                                    if (kATmem)
                                        umma_ts<KIND>(tmem + (uint32_t)(l * kBN), tmem + (uint32_t)(kACol + sa * 8),
                                                      db + (uint64_t)((sb * kBTile) >> 4), idesc,
                                                      sa == 0 ? first : 1u);
                                    else
                                        umma<KIND>(tmem + (uint32_t)(l * kBN),
                                                   da + (uint64_t)((sa * kATile) >> 4),
                                                   db + (uint64_t)((sb * kBTile) >> 4), idesc,
                                                   sa == 0 ? first : 1u);
                                }
                            }
                            umma_commit(&empty_bar[st]);       // frees the stage when these MMAs finish
                            if (++st == stages) { st = 0; ph ^= 1; }
                        }
                        umma_commit(&accf_bar);                // accumulators ready for the epilogue
                        ndrain++;
                    }
                }
            }
            if (!ok) {
                abort_s = 1;
                atomicExch(err, 7);
                // the MMAs already issued must finish before TMEM is freed
                volatile int never = 0;
                umma_commit(&drain_bar);
                (void)mbar_wait(&drain_bar, 0, &never, kWaitNs);
            }
        }
    } else {
        // ------------------------------------------------ epilogue (warps 0-3)
        const int row = warp * 32 + lane;                 // TMEM lane == tile row
        const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
        uint32_t accph = 0;
        bool ok = true;
        double lw[S];                                     // 2^(-beta * l)
        lw[0] = 1.0;
#pragma unroll
        for (int l = 1; l < S; l++) lw[l] = ldexp(lw[l - 1], -beta);
        for (int it = blockIdx.x; it < nitems && ok; it += gridDim.x) {
            const DItem item = items[it];
            const DCBlock &cb = cblks[item.cblk];
            double acc[kBN];
#pragma unroll
            for (int j = 0; j < kBN; j++) acc[j] = 0.0;
            const int m = item.m0 + row;
            for (int ti = cb.t_begin; ti < cb.t_end && ok; ti++) {
                const DOzTask t = tasks[ti];
                const DPanel &pa = panels[t.pa];
                const DPanel &pb = panels[t.pb];
                const int nkb = pa.K_pad / kbe;
                const double f = ldexp(t.coeff, exps[pa.exp_off + m] - 2 * beta0);
                const int32_t *eb = exps + pb.exp_off + item.n0;
                for (int kb0 = 0; kb0 < nkb; kb0 += chunk_kb) {
                    // warp-uniform outcome: tcgen05.ld below is .sync.aligned
                    ok = __all_sync(0xffffffffu, mbar_wait(&accf_bar, accph, &abort_s, wait_ns));
                    if (!ok) break;
                    accph ^= 1;
                    tc_fence_after();
#pragma unroll
                    for (int c = 0; c < kBN / 8; c++) {
                        uint32_t v[S][8];
#pragma unroll
                        for (int l = 0; l < S; l++) tmem_ld8(lane_base + (uint32_t)(l * kBN + c * 8), v[l]);
                        tmem_wait_ld();
#pragma unroll
                        for (int j = 0; j < 8; j++) {
                            double sum = 0.0;
#pragma unroll
                            for (int l = S - 1; l >= 0; l--) {
                                const double x = KIND == kOzInt8 ? (double)(int32_t)v[l][j]
                                                                 : (double)__uint_as_float(v[l][j]);
                                sum += lw[l] * x;
                            }
                            acc[c * 8 + j] += ldexp(f, eb[c * 8 + j]) * sum;
                        }
                    }
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&acce_bar);
                }
            }
            if (!ok) break;
            // FP64 write of the finished tile row
            if constexpr (SCATTER) {
                if (m < cb.M) {
                    const int2 dr = drange[item.cblk];
                    for (int d = dr.x; d < dr.y; d++) {
                        const DCBlock &db = dests[d];
                        const int64_t drow = db.c_off + mixed_offset(m, db.nm, db.mext, db.mc_str);
#pragma unroll
                        for (int j = 0; j < kBN; j++) {
                            const int n = item.n0 + j;
                            if (n < cb.N)
                                atomicAdd(Cp + drow + mixed_offset(n, db.nn, db.next, db.nc_str), db.scale * acc[j]);
                        }
                    }
                }
            } else if (m < cb.M) {
                const int64_t orow = cb.c_off + mixed_offset(m, cb.nm, cb.mext, cb.mc_str);
#pragma unroll
                for (int j = 0; j < kBN; j++) {
                    const int n = item.n0 + j;
                    if (n < cb.N) {
                        double *dst = Cp + orow + mixed_offset(n, cb.nn, cb.next, cb.nc_str);
                        const double v = cb.scale * acc[j];
                        if (add) *dst += v;
                        else *dst = v;
                    }
                }
            }
        }
        if (!ok) { abort_s = 1; atomicExch(err, 7); }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" :: "r"(tmem) : "memory");
    }
}

int g_nsm = 0;

template<int KIND, int S, bool SCATTER = false>
cudaError_t launch_gemm_s(const DPanel *panels, const uint8_t *slices, const DOzTask *tasks, const DCBlock *cblks,
                          const DItem *items, int32_t nitems, const int32_t *exps, double *c, int32_t add,
                          int32_t chunk_kb, int32_t *err, uint64_t wait_ns, cudaStream_t s,
                          const int2 *drange = nullptr, const DCBlock *dests = nullptr) {
    int beta0, beta, esz, kbe;
    int64_t mp;
    oz_kind_params(KIND, &beta0, &beta, &esz, &kbe, &mp);
    constexpr int stage_bytes = S * (kATile + kBTile);
    int stages = (200 * 1024) / stage_bytes;
    if (stages > kMaxStages) stages = kMaxStages;
    if (stages < 2) return cudaErrorInvalidValue;
    // At least 120 KB so that a second CTA never shares the SM: each CTA
    // holds all 512 TMEM columns.
    size_t smem = (size_t)stages * stage_bytes + 1024;
    if (smem < 120 * 1024) smem = 120 * 1024;
    cudaError_t e = cudaFuncSetAttribute(oz_gemm_kernel<KIND, S, SCATTER>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (g_nsm == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_nsm, cudaDevAttrMultiProcessorCount, dev);
    }
    int grid = nitems < g_nsm ? nitems : g_nsm;
    if (grid < 1) return cudaSuccess;
    oz_gemm_kernel<KIND, S, SCATTER><<<grid, kThreads, smem, s>>>(panels, slices, tasks, cblks, items, nitems, exps,
                                                                 c, add, stages, chunk_kb, beta0, beta, kbe, err,
                                                                 wait_ns, drange, dests);
    return cudaGetLastError();
}

template<int KIND>
cudaError_t launch_gemm_k(int S, const DPanel *panels, const uint8_t *slices, const DOzTask *tasks,
                          const DCBlock *cblks, const DItem *items, int32_t nitems, const int32_t *exps, double *c,
                          int32_t add, int32_t chunk_kb, int32_t *err, uint64_t wait_ns, cudaStream_t s) {
    switch (S) {
#define CASE_S(n) case n: return launch_gemm_s<KIND, n>(panels, slices, tasks, cblks, items, nitems, exps, c, add, chunk_kb, err, wait_ns, s);
    CASE_S(1) CASE_S(2) CASE_S(3) CASE_S(4) CASE_S(5) CASE_S(6) CASE_S(7) CASE_S(8)
#undef CASE_S
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t launch_oz_split(int kind, const DPanel *panels, int32_t npanels, int32_t max_rows_pad,
                            const double *a, const double *b, uint8_t *slices, int32_t *exps,
                            int32_t S, cudaStream_t s) {
    if (npanels <= 0) return cudaSuccess;
    int beta0, beta, esz, kbe;
    int64_t mp;
    oz_kind_params(kind, &beta0, &beta, &esz, &kbe, &mp);
    dim3 grid((max_rows_pad + 31) / 32, npanels < 65535 ? npanels : 65535);
    if (kind == kOzInt8)
        oz_split_kernel<kOzInt8><<<grid, 256, 0, s>>>(panels, npanels, a, b, slices, exps, S, beta0, beta);
    else if (kind == kOzBf16)
        oz_split_kernel<kOzBf16><<<grid, 256, 0, s>>>(panels, npanels, a, b, slices, exps, S, beta0, beta);
    else
        oz_split_kernel<kOzE4m3><<<grid, 256, 0, s>>>(panels, npanels, a, b, slices, exps, S, beta0, beta);
    return cudaGetLastError();
}

cudaError_t launch_oz_gemm(int kind, const DPanel *panels, const uint8_t *slices, const DOzTask *tasks,
                           const DCBlock *cblks, const DItem *items, int32_t nitems, const int32_t *exps,
                           double *c, int32_t add, int32_t S, int32_t chunk_kb, int32_t *err,
                           uint64_t wait_ns, cudaStream_t s, const int2 *drange, const DCBlock *dests) {
    if (S < 1 || S > 8) return cudaErrorInvalidValue;
    if (dests) {
        // the scattering form for each kind's default slice count only
        if (kind == kOzInt8 && S == 7)
            return launch_gemm_s<kOzInt8, 7, true>(panels, slices, tasks, cblks, items, nitems, exps, c, 0, chunk_kb,
                                                   err, wait_ns, s, drange, dests);
        if (kind == kOzBf16 && S == 7)
            return launch_gemm_s<kOzBf16, 7, true>(panels, slices, tasks, cblks, items, nitems, exps, c, 0, chunk_kb,
                                                   err, wait_ns, s, drange, dests);
        if (kind == kOzE4m3 && S == 8)
            return launch_gemm_s<kOzE4m3, 8, true>(panels, slices, tasks, cblks, items, nitems, exps, c, 0, chunk_kb,
                                                   err, wait_ns, s, drange, dests);
        return cudaErrorNotSupported;
    }
    if (kind == kOzInt8)
        return launch_gemm_k<kOzInt8>(S, panels, slices, tasks, cblks, items, nitems, exps, c, add, chunk_kb, err,
                                      wait_ns, s);
    if (kind == kOzBf16)
        return launch_gemm_k<kOzBf16>(S, panels, slices, tasks, cblks, items, nitems, exps, c, add, chunk_kb, err,
                                      wait_ns, s);
    return launch_gemm_k<kOzE4m3>(S, panels, slices, tasks, cblks, items, nitems, exps, c, add, chunk_kb, err,
                                  wait_ns, s);
}

}  // namespace ltg
