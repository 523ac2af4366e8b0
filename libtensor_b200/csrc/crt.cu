// Modular (CRT) split-precision contraction on the tcgen05 INT8 tensor cores.
//
// FP64 operands are scaled row by row to integers of P bits and multiplied
// exactly as their residues modulo L pairwise coprime moduli m_l <= 256
// (the "integer modular" emulation of Ozaki, Uchino and Imamura, 2024):
//   1. exponents (crt_exp_kernel): for every operand row, the exponent of its
//      largest magnitude, combined over all panels that feed the same global
//      row of C (atomicMax into one table per side of C), so that every pair
//      of a C block shares the row and column scaling.  Long rows may be
//      sampled instead (one 32-element run in kSampleGroups, one binade of
//      headroom): the residue pass then forms their exact maxima as it reads
//      them, and rows whose sampled bound was too small are redone with the
//      exact exponent (see crt_res_kernel);
//   2. residues (crt_res_kernel): X = c_p * rint(x * 2^(P - e_row)) (the
//      pair's integer coefficient c_p folded in on one side), stored as its
//      balanced residues mod m_l (INT8) in shared-memory tile images;
//   3. products (crt_gemm_kernel): per C tile and modulus, all pairs and k
//      blocks accumulate sum_p sum_k A_l * B_l exactly in one INT32 TMEM
//      accumulator (|sum| < 2^31 is checked on the host); the epilogue warps
//      reduce it mod m_l to one byte per element; items of one 128-row tile
//      alternate between two accumulator slots, so that the MMA warp fills
//      one with the next modulus while the epilogue drains the other;
//   4. recombination (crt_combine_kernel): Garner's mixed-radix algorithm
//      with balanced digits gives the exact integer sum_p c_p A'_p B'_p in
//      (-M/2, M/2), M = prod m_l (the host chooses P so that it fits), which
//      is scaled by 2^(e_row + e_col - 2P) and the contraction coefficient in
//      FP64 and written to C (assign or add).
// The error is that of rounding each operand to P bits relative to its row's
// largest element (P about 43 for 13 moduli and K up to a few thousand).
//
// Warp roles of the products kernel (320 threads): warps 0-7 epilogue (two
// per TMEM lane quarter, one tile row per thread, alternate 16-column
// chunks), warp 8 bulk-copy producer, warp 9 MMA issuer.  Operand tiles are whole tile images moved by 1-D
// cp.async.bulk (no tensor maps, no multicast); every mbarrier wait is
// bounded in time and reports through *err.
#include <type_traits>

#include "ltg_device.cuh"


namespace ltg {
namespace {

constexpr int kXRows = 128;                         // MMA M (TMEM lanes)
constexpr int kKB = 32;                             // bytes (INT8 elements) per k block
constexpr int kXTile = kXRows * kKB;                // 4 KB
constexpr int kMaxNt = 256;
constexpr int kSubBytes = 2 * kXTile + kMaxNt * kKB;    // one k block: two M tiles and one N tile (16 KB)
// (a stage holds KB k blocks as [M tile 0][M tile 1][N tile] regions; KB is
// the products kernel's template parameter, crt_stage_kb() at launch)
constexpr int kMaxStages = 8;
constexpr int kEpiWarps = 8;                        // two per TMEM lane quarter
constexpr int kGemmThreads = 32 * (kEpiWarps + 2);  // + bulk-copy producer + MMA issuer
constexpr uint64_t kWaitNs = 2000000000ull;         // 2 s: the drain waits after an abort
constexpr double kMagicD = 6755399441055744.0;      // 1.5 * 2^52: round-to-integer constant
constexpr float kMagicF = 12582912.0f;              // 1.5 * 2^23
constexpr int32_t kNoExp = -1000000;                // exponent of a row with no non-zero element

// The moduli (pairwise coprime, <= 256) and the constants derived from them,
// as compile-time functions so that unrolled loops over the moduli fold them
// into instruction operands.  The same list is used by the host
// (kCrtModuli in ltg_capi.cu).
__host__ __device__ constexpr int32_t crt_modulus(int i) {
    return i == 0 ? 256 : i == 1 ? 255 : i == 2 ? 253 : i == 3 ? 251 : i == 4 ? 247 : i == 5 ? 241 :
           i == 6 ? 239 : i == 7 ? 233 : i == 8 ? 229 : i == 9 ? 227 : i == 10 ? 223 : i == 11 ? 217 :
           i == 12 ? 211 : i == 13 ? 199 : i == 14 ? 197 : 193;
}
// m_j^-1 mod m_i (extended Euclid)
__host__ __device__ constexpr int32_t crt_inverse(int j, int i) {
    int64_t m = crt_modulus(i), t = 0, nt = 1, r = m, nr = crt_modulus(j) % m;
    while (nr != 0) {
        const int64_t q = r / nr;
        const int64_t t2 = t - q * nt; t = nt; nt = t2;
        const int64_t r2 = r - q * nr; r = nr; nr = r2;
    }
    return (int32_t)(t < 0 ? t + m : t);
}

// Balanced representative of x mod m, in (-m/2, m/2].
__host__ __device__ constexpr int32_t crt_balanced(int64_t x, int32_t m) {
    const int64_t y = ((x % m) + m) % m;
    return (int32_t)(y > m / 2 ? y - m : y);
}
__host__ __device__ constexpr bool crt_odd_moduli() {
    for (int i = 1; i < 16; i++)
        if (crt_modulus(i) % 2 == 0) return false;
    return true;
}
static_assert(crt_odd_moduli(), "the single-reduction Garner digits need odd moduli after m_0");
// Garner's digit i as one linear form: the recurrence t <- (t - v_j) m_j^-1
// (mod m_i), j = 0..i-1, started at t = r_i, expands to
//   v_i = r_i * prod_{j<i} m_j^-1 - sum_{j<i} v_j * prod_{k=j..i-1} m_k^-1  (mod m_i),
// so the digit costs i multiply-adds and one reduction.  The products are
// taken balanced (|.| <= 128).
__host__ __device__ constexpr int32_t crt_garner_d(int j, int i) {
    int64_t p = 1;
    for (int k = j; k < i; k++) p = p * crt_inverse(k, i) % crt_modulus(i);
    return crt_balanced(p, crt_modulus(i));
}

// Compile-time loop: f(std::integral_constant<int, I>) for I in [B, E).
template<int B, int E>
struct StaticFor {
    template<class F>
    __device__ __forceinline__ static void run(F &&f) {
        f(std::integral_constant<int, B>());
        StaticFor<B + 1, E>::run(f);
    }
};
template<int E>
struct StaticFor<E, E> {
    template<class F>
    __device__ __forceinline__ static void run(F &&) {}
};

__device__ __forceinline__ int64_t mixed_offset(int32_t lin, int n, const int32_t *ext, const int32_t *str) {
    int64_t off = 0;
    for (int i = n - 1; i >= 0; i--) {
        const int32_t e = ext[i];
        const int32_t q = lin / e;
        off += (int64_t)(lin - q * e) * str[i];
        lin = q;
    }
    return off;
}

// Byte offset of element (row r, k byte kb_byte of k block kb) of modulus l
// in a panel's tile images: [row tile][modulus][k block] images of TR rows x
// 32 bytes (so that the k blocks of one pipeline stage are one contiguous
// copy), K-major core matrices of 8 rows x 16 bytes (the two 16-byte k halves
// 128 bytes apart, 8-row groups 256 bytes apart).
__device__ __forceinline__ int64_t image_offset(int r, int TR, int nkb, int kb, int l, int L, int kb_byte) {
    const int tile = r / TR, rr = r - tile * TR;
    return ((int64_t)(tile * L + l) * nkb + kb) * (int64_t)(TR * kKB) + (rr >> 3) * 256 +
           (kb_byte >> 4) * 128 + (rr & 7) * 16 + (kb_byte & 15);
}

// ---------------------------------------------------------------- split passes
//
// Work units (built on the host): rows [r0, r0 + nrows) of one panel, all of
// its k, in one of two thread mappings:
//  - rows (long k): 32 rows, 8 threads per row, each reading 4 consecutive k
//    per step along the row; the row maximum is reduced over the 8 threads;
//  - tiles (short k, e.g. the cells of grouped products): core tiles of 8 rows
//    x 16 k, the shape of one 128-byte core matrix of a residue image (lane l
//    takes row l / 4 and the 4 consecutive k of group l % 4), spread over the
//    CTA's warps, so that short rows still fill the warps.
// When a panel's k dims are not one contiguous run, their offsets come from a
// shared-memory table built once per unit (no divisions per element).

constexpr int kSplitThreads = 256;
constexpr int kSplitWarps = kSplitThreads / 32;
constexpr int kKoffMax = 4096;                      // k offsets tabulated per unit
constexpr int kUnitRowsMax = 256;                   // rows per unit (bound of the host's units)
constexpr int kUnitRowMap = 0, kUnitTileMap = 1;    // thread mapping of a unit (units[].w)
// Sampled exponents: rows of row-mapped units with at least kSampleMinK
// k words read one 32-element run in kSampleGroups (the 8 threads of the
// row one 4-element group each, so that a run is one 256-byte read) for
// their bound.
constexpr int kSampleMinK = 1024;
constexpr int kSampleGroups = 16;
__host__ __device__ __forceinline__ bool sampled_panel(const DCrtPanel &P, int unit_map) {
    return unit_map == kUnitRowMap && P.wk >= kSampleMinK;
}

__global__ void crt_fill_kernel(int32_t *p, int32_t n, int32_t v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}


// k offset mode of a panel: 0 contiguous, 1 tabulated in koff, 2 computed.
__device__ __forceinline__ int koff_setup(const DCrtPanel &P, int32_t *koff) {
    const int mode = (P.nk == 1 && P.kstr[0] == 1) ? 0 : (P.K <= kKoffMax ? 1 : 2);
    if (mode == 1)
        for (int k = threadIdx.x; k < P.K; k += blockDim.x) koff[k] = (int32_t)mixed_offset(k, P.nk, P.kext, P.kstr);
    return mode;
}
__device__ __forceinline__ int64_t koffset(const DCrtPanel &P, int mode, const int32_t *koff, int k) {
    return mode == 0 ? k : (mode == 1 ? koff[k] : mixed_offset(k, P.nk, P.kext, P.kstr));
}

__global__ void __launch_bounds__(kSplitThreads)
crt_exp_kernel(const DCrtPanel *__restrict__ panels, const int4 *__restrict__ units, int32_t nunits,
               const double *__restrict__ A, const double *__restrict__ B, const int32_t *__restrict__ gidx,
               int32_t *ex, int32_t *ey, int32_t sample) {
    __shared__ int32_t koff[kKoffMax];
    __shared__ int32_t rexp[kUnitRowsMax];
    __shared__ int64_t roff[kUnitRowsMax];                  // tile mapping: the unit's row offsets
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, lrow = lane >> 2, kq = lane & 3;
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const int4 un = units[u];
        const DCrtPanel &P = panels[un.x];
        // shared memory is used by tabulated k offsets and the tile mapping
        // (both uniform over the CTA); the first barrier keeps the previous
        // unit's readers (a grid smaller than the unit count) apart
        const bool shared = (P.nk != 1 || P.kstr[0] != 1) || un.w == kUnitTileMap;
        if (shared) __syncthreads();
        const int mode = koff_setup(P, koff);
        if (un.w == kUnitTileMap)
            for (int i = threadIdx.x; i < un.z; i += blockDim.x) {
                rexp[i] = kNoExp;
                roff[i] = un.y + i < P.rows ? mixed_offset(un.y + i, P.nr, P.rext, P.rstr) : 0;
            }
        if (shared) __syncthreads();
        const double *src = (P.src ? B : A) + P.src_off;
        int32_t *tab = P.side == 0 ? ex : ey;
        if (un.w == kUnitRowMap) {
            const int lr = threadIdx.x >> 3, c = threadIdx.x & 7;
            const int r = un.y + lr;
            const bool valid = lr < un.z && r < P.rows;
            const double *row = src + (valid ? mixed_offset(r, P.nr, P.rext, P.rstr) : 0);
            // sampled: group c of every kSampleGroups-th run of 32 elements;
            // else group c of every run
            const bool smp = sample && sampled_panel(P, un.w);
            const int step = smp ? 32 * kSampleGroups : 32, first = 4 * c;
            double mx = 0.0;
            if (valid)
                for (int k0 = first; k0 < P.K; k0 += step)
#pragma unroll
                    for (int j = 0; j < 4; j++)
                        if (k0 + j < P.K) mx = fmax(mx, fabs(row[koffset(P, mode, koff, k0 + j)]));
            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 2));
            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 4));
            if (valid && c == 0 && mx > 0.0) {
                int e;
                frexp(mx, &e);
                atomicMax(&tab[gidx[P.g_off + r]], smp ? e + 1 : e);   // one binade of headroom
            }
            continue;
        }
        const int nkt = (P.K + 15) >> 4;
        const int ntile = ((un.z + 7) >> 3) * nkt;
        for (int t = warp; t < ntile; t += kSplitWarps) {
            const int rg = t / nkt, kt = t - rg * nkt;
            const int rl = rg * 8 + lrow, r = un.y + rl;
            const bool valid = rl < un.z && r < P.rows;
            double mx = 0.0;
            if (valid) {
                const double *row = src + roff[rl];
                const int k0 = kt * 16 + kq * 4;
#pragma unroll
                for (int j = 0; j < 4; j++)
                    if (k0 + j < P.K) mx = fmax(mx, fabs(row[koffset(P, mode, koff, k0 + j)]));
            }
            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 2));
            if (valid && kq == 0 && mx > 0.0) {
                int e;
                frexp(mx, &e);                                 // mx = f * 2^e, f in [0.5, 1)
                atomicMax(&rexp[rl], e);
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < un.z; i += blockDim.x) {
            const int r = un.y + i;
            if (r < P.rows && rexp[i] > kNoExp) atomicMax(&tab[gidx[P.g_off + r]], rexp[i]);
        }
    }
}

// ---------------------------------------------------------------- residues

// Residue of an integer X (|X| < 2^51, given as a double and as its low 32
// bits) modulo m, as the low byte of X - m * rint(X / m).  The quotient
// rint(X * (1/m)) comes out of one FMA against the 1.5 * 2^52 constant (its
// low word is q mod 2^32) and is exact: the product's relative error 2^-53
// moves X/m by less than 2^-10.5, while X/m mod 1 stays at least 1/(2m) away
// from 1/2 for odd m, and the scaling is exact for m = 256.  So the balanced
// residue r = X - q m lies in [-(m-1)/2, (m-1)/2] (or is +-128 for m = 256,
// where both share the byte 0x80), and its low byte is (X - q m) mod 2^8,
// formed in 32-bit integer arithmetic.
template<int I>
__device__ __forceinline__ uint32_t residue_byte(double X, uint32_t xlo) {
    constexpr double minv = 1.0 / (double)crt_modulus(I);
    const uint32_t qlo = (uint32_t)__double2loint(fma(X, minv, kMagicD));
    return xlo - qlo * (uint32_t)crt_modulus(I);
}

// Low bytes of four words packed into one.
__device__ __forceinline__ uint32_t pack4(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    return __byte_perm(__byte_perm(a, b, 0x0040), __byte_perm(c, d, 0x0040), 0x5410);
}

// Sampled rows (sampled_panel): their residues are formed with the sampled
// bound e (|x| < 2^e unless the sample missed the row's largest elements),
// and the row's exact exponent goes to the side's second table (ext / eyt).
// With redo set, only those rows run again, and only where the exact
// exponent exceeds the bound: with the exact exponent, overwriting the
// residues formed before (whose integers may have exceeded 2^P).
template<int L>
__global__ void __launch_bounds__(kSplitThreads, 4)
crt_res_kernel(const DCrtPanel *__restrict__ panels, const int4 *__restrict__ units, int32_t nunits,
               const double *__restrict__ A, const double *__restrict__ B, const int32_t *__restrict__ gidx,
               const int32_t *__restrict__ ex, const int32_t *__restrict__ ey, int32_t *ext, int32_t *eyt,
               int32_t sample, int32_t redo, uint8_t *__restrict__ res, const CrtParams cp) {
    __shared__ int32_t koff[kKoffMax];
    __shared__ int64_t roff[kUnitRowsMax];                  // tile mapping: the unit's row offsets
    __shared__ int32_t rexp[kUnitRowsMax];                  //   and exponents
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, lrow = lane >> 2, kq = lane & 3;
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const int4 un = units[u];
        const DCrtPanel &P = panels[un.x];
        // tabulated k offsets and the tile mapping's row tables (uniform)
        const bool shared = P.nk != 1 || P.kstr[0] != 1 || (un.w == kUnitTileMap && !redo);
        if (shared) __syncthreads();                         // the previous unit's readers are done
        const int mode = koff_setup(P, koff);
        if (un.w == kUnitTileMap && !redo)
            for (int i = threadIdx.x; i < un.z; i += blockDim.x) {
                const int r = un.y + i;
                const bool valid = r < P.rows;
                roff[i] = valid ? mixed_offset(r, P.nr, P.rext, P.rstr) : 0;
                rexp[i] = valid ? (P.side == 0 ? ex : ey)[gidx[P.g_off + r]] : kNoExp;
            }
        if (shared) __syncthreads();
        const double *src = (P.src ? B : A) + P.src_off;
        const int32_t *tab = P.side == 0 ? ex : ey;
        int32_t *tabt = P.side == 0 ? ext : eyt;
        uint8_t *base = res + P.res_off;
        const int TR = P.tr, nkb = P.K_pad / kKB;
        const double coef = (double)P.coef;
        const int64_t lstride = (int64_t)nkb * TR * kKB;      // the same k block of the next modulus
        int cur = -1;
        const double *row = src;
        double s1 = 0.0, s2 = 0.0;
        bool live = false, rowok = false, fast = false, vec = false;
        // row r's offset and scaling (exponent e_over, or the side table's;
        // the tile mapping passes both from its row tables), kept while the
        // thread stays on it
        auto set_row = [&](int r, int e_over, int64_t off = -1) {
            cur = r;
            const bool valid = r < P.rows;
            row = src + (!valid ? 0 : off >= 0 ? off : mixed_offset(r, P.nr, P.rext, P.rstr));
            const int e = !valid ? kNoExp : (e_over > kNoExp ? e_over : tab[gidx[P.g_off + r]]);
            // 2^(P - e) as two finite factors
            const int sh = e > kNoExp ? cp.P - e : 0;
            s1 = ldexp(1.0, sh / 2);
            s2 = ldexp(1.0, sh - sh / 2);
            live = valid && e > kNoExp;
            rowok = valid;
            vec = mode == 0 && ((uintptr_t)row & 15) == 0;
            // one finite factor and no coefficient: one FMA forms the integer
            fast = sh <= 1000 && P.coef == 1;
            if (fast) { s1 = ldexp(1.0, sh); s2 = 1.0; }
        };
        // elements k0..k0+3 of the current row (zero past K, and zero for a
        // row without elements unless any: a sampled row's exact maximum is
        // formed from them, and a non-zero row whose bound said "no element"
        // is redone)
        auto load4_if = [&](int k0, double *x, bool any) {
            const bool ok = any ? rowok : live;
            if (ok && vec && k0 + 3 < P.K) {
                // contiguous, 16-byte aligned row: two 16-byte loads
                const double2 a = *reinterpret_cast<const double2 *>(row + k0);
                const double2 b = *reinterpret_cast<const double2 *>(row + k0 + 2);
                x[0] = a.x; x[1] = a.y; x[2] = b.x; x[3] = b.y;
                return;
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int k = k0 + j;
                x[j] = (ok && k < P.K) ? row[koffset(P, mode, koff, k)] : 0.0;
            }
        };
        // residues of k0..k0+3 of row r (k0 % 4 == 0) into the images; the
        // fast form (fast_c true: one scale factor, coefficient 1) needs the
        // row's fast flag
        auto put4g = [&](auto fast_c, int r, int k0, const double *x) {
            constexpr bool kFast = decltype(fast_c)::value;
            uint32_t packed[L];
#pragma unroll
            for (int l = 0; l < L; l++) packed[l] = 0;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                double tt, X;
                uint32_t xlo;                                         // X mod 2^32
                if (kFast) {
                    tt = fma(x[j], s1, kMagicD);                      // 1.5 * 2^52 + rint(x 2^(P-e))
                    X = tt - kMagicD;
                    xlo = (uint32_t)__double2loint(tt);
                } else {
                    tt = (x[j] * s1) * s2 + kMagicD;
                    X = (tt - kMagicD) * coef;                        // the integer coefficient folded in
                    xlo = (uint32_t)__double2loint(tt) * (uint32_t)P.coef;
                }
                // byte j of each modulus word takes this element's residue
                const uint32_t sel = 0x3210u ^ ((0x4u ^ (uint32_t)j) << (4 * j));
                StaticFor<0, L>::run([&](auto ic) {
                    constexpr int l = decltype(ic)::value;
                    packed[l] = __byte_perm(packed[l], residue_byte<l>(X, xlo), sel);
                });
            }
            const int kk = P.k0 + k0;                                // a multiple of 4: one word
            uint8_t *dst0 = base + image_offset(P.r0 + r, TR, nkb, kk / kKB, 0, L, kk % kKB);
#pragma unroll
            for (int l = 0; l < L; l++) *reinterpret_cast<uint32_t *>(dst0 + l * lstride) = packed[l];
        };
        auto put4 = [&](int r, int k0) {
            double x[4];
            load4_if(k0, x, false);
            put4g(std::false_type(), r, k0, x);
        };
        if (un.w == kUnitRowMap) {
            const int lr = threadIdx.x >> 3, c = threadIdx.x & 7;
            const int r = un.y + lr;
            const bool smp = sample && sampled_panel(P, un.w);       // uniform over the CTA
            if (redo && !smp) continue;
            const bool rv = lr < un.z && r < P.wrows;
            // largest |x| of the row as the largest high word without its
            // sign bit (ordered as |x|; its exponent field is that of the maximum)
            uint32_t mx = 0;
            if (rv) {
                bool act = true;
                int e_over = kNoExp;
                if (redo) {
                    // the exact exponent against the bound the residues used
                    const int g = gidx[P.g_off + r];
                    e_over = tabt[g];
                    act = e_over > tab[g];
                }
                if (act) {
                    set_row(r, e_over);
                    const bool track = smp && !redo;
                    auto run = [&](auto fast_c) {
                        for (int k0 = 4 * c; k0 < P.wk; k0 += 32) {
                            double x[4];
                            load4_if(k0, x, track);
                            if (track)
#pragma unroll
                                for (int j = 0; j < 4; j++)
                                    mx = max(mx, (uint32_t)__double2hiint(x[j]) & 0x7fffffffu);
                            put4g(fast_c, r, k0, x);
                        }
                    };
                    if (fast) run(std::true_type());
                    else run(std::false_type());
                }
            }
            if (smp && !redo) {
                // the row's exact exponent (all 8 threads of every row of the warp take part)
                mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
                mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, 2));
                mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, 4));
                if (rv && c == 0 && mx != 0) {
                    // frexp's exponent of a normal number with biased exponent b is
                    // b - 1022; subnormals (b = 0) take -1022, above their own
                    const int b = (int)(mx >> 20);
                    atomicMax(&tabt[gidx[P.g_off + r]], (b > 0 ? b : 1) - 1022);
                }
            }
            continue;
        }
        if (redo) continue;                                  // tile-mapped units read every element
        const int nkt = (P.wk + 15) >> 4;
        const int ntile = ((un.z + 7) >> 3) * nkt;
        for (int t = warp; t < ntile; t += kSplitWarps) {
            const int rg = t / nkt, kt = t - rg * nkt;
            const int rl = rg * 8 + lrow, r = un.y + rl;
            const int k0 = kt * 16 + kq * 4;
            if (rl >= un.z || r >= P.wrows || k0 >= P.wk) continue;
            if (r != cur) set_row(r, rexp[rl], roff[rl]);
            put4(r, k0);
        }
    }
}

// ---------------------------------------------------------------- fused split of row families
//
// The two passes above read every operand element twice from HBM (once for
// the row maxima, once for the residues).  For a row family (DCrtFamily) the
// exponent of a row needs only that family's rows, so one CTA splits a unit
// of kFuseRows rows of a family completely: pass 1 reads the rows (all of the
// family's k) and forms their maxima, pass 2 reads them again -- from L2:
// the resident CTAs hold kFuseRows rows of a family each, tens of MB in all
// -- and writes the residue images.  HBM then sees the operand once.  Lane
// mapping of both passes: kFuseRows rows x 16 groups of 4 consecutive k per
// warp (a 64-wide k tile), so that pass-2 stores of a warp fill whole
// 32-byte sectors of the core matrices (two rows x 16 bytes each).  Family
// panels have one contiguous k run (k offset = k).

// Shapes of the one-read split (rows per unit, threads, CTAs per SM); the
// resident CTAs' rows must stay well inside L2 (148 SMs x CTAs x rows x the
// family's k x 8 bytes).
template<int ROWS, int THREADS, int MINB>
struct FuseCfg {
    static constexpr int kRows = ROWS, kThreads = THREADS, kCtasPerSm = MINB;
    static constexpr int kWarps = THREADS / 32;
    static constexpr int kLanesPerRow = 32 / ROWS;     // 4-k groups per row in a warp tile
    static constexpr int kTileK = 4 * kLanesPerRow;    // k per warp tile
};

template<int L, class FC>
__global__ void __launch_bounds__(FC::kThreads, FC::kCtasPerSm)
crt_fused_kernel(const DCrtPanel *__restrict__ panels, const DCrtFamily *__restrict__ fams,
                 const int32_t *__restrict__ famp, const int32_t *__restrict__ famt,
                 const int4 *__restrict__ units, int32_t nunits, const double *__restrict__ A,
                 const double *__restrict__ B, const int32_t *__restrict__ gidx, int32_t *ex, int32_t *ey,
                 uint8_t *__restrict__ res, const CrtParams cp) {
    __shared__ int32_t rexp[FC::kRows];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int lrow = lane / FC::kLanesPerRow, kq = lane % FC::kLanesPerRow;
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const int4 un = units[u];
        const DCrtFamily F = fams[un.x];
        __syncthreads();                                       // the previous unit's readers of rexp are done
        if (threadIdx.x < FC::kRows) rexp[threadIdx.x] = kNoExp;
        __syncthreads();
        const int r = un.y + lrow;
        const bool rvalid = lrow < un.z;
        // pass 1: row maxima, panel by panel (a lane keeps one row: a running
        // maximum over its tiles, reduced once)
        double mx = 0.0;
        if (rvalid) {
            for (int q = F.p_begin; q < F.p_end; q++) {
                const DCrtPanel &P = panels[famp[q]];
                const double *row = (P.src ? B : A) + P.src_off + mixed_offset(r, P.nr, P.rext, P.rstr);
                const int nt = (P.K + FC::kTileK - 1) / FC::kTileK;
#pragma unroll 4
                for (int t = warp; t < nt; t += FC::kWarps) {
                    const int k0 = t * FC::kTileK + kq * 4;
#pragma unroll
                    for (int j = 0; j < 4; j++)
                        if (k0 + j < P.K) mx = fmax(mx, fabs(row[k0 + j]));
                }
            }
        }
#pragma unroll
        for (int o = 1; o < FC::kLanesPerRow; o <<= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (rvalid && kq == 0 && mx > 0.0) {
            int e;
            frexp(mx, &e);                                     // mx = f * 2^e, f in [0.5, 1)
            atomicMax(&rexp[lrow], e);
        }
        __syncthreads();
        if (threadIdx.x < un.z) {
            const DCrtPanel &P0 = panels[famp[F.p_begin]];
            int32_t *tab = P0.side == 0 ? ex : ey;
            tab[gidx[P0.g_off + un.y + threadIdx.x]] = rexp[threadIdx.x];
        }
        if (!rvalid) continue;
        // pass 2: residues (the reads hit L2)
        const int e = rexp[lrow];
        const int sh = e > kNoExp ? cp.P - e : 0;
        const double s1 = ldexp(1.0, sh / 2), s2 = ldexp(1.0, sh - sh / 2);   // 2^(P - e), two finite factors
        const bool live = e > kNoExp;
        for (int q = F.p_begin; q < F.p_end; q++) {
            const DCrtPanel &P = panels[famp[q]];
            const double *row = (P.src ? B : A) + P.src_off + mixed_offset(r, P.nr, P.rext, P.rstr);
            const double coef = (double)P.coef;
            const uint32_t icoef = (uint32_t)P.coef;
            const int nkb = P.K_pad / kKB;
            const int64_t lstride = (int64_t)nkb * P.tr * kKB;  // the same k block of the next modulus
            uint8_t *pbase = res + P.res_off;
            const int nt = (P.wk + FC::kTileK - 1) / FC::kTileK;
            for (int t = warp; t < nt; t += FC::kWarps) {
                const int k0 = t * FC::kTileK + kq * 4;
                if (k0 >= P.wk) continue;
                double x[4];
#pragma unroll
                for (int j = 0; j < 4; j++) x[j] = (live && k0 + j < P.K) ? row[k0 + j] : 0.0;
                uint32_t packed[L];
#pragma unroll
                for (int l = 0; l < L; l++) packed[l] = 0;
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const double tt = (x[j] * s1) * s2 + kMagicD;         // 1.5 * 2^52 + rint(x 2^(P-e))
                    const double X = (tt - kMagicD) * coef;               // the integer coefficient folded in
                    const uint32_t xlo = (uint32_t)__double2loint(tt) * icoef;   // X mod 2^32
                    const uint32_t sel = 0x3210u ^ ((0x4u ^ (uint32_t)j) << (4 * j));
                    StaticFor<0, L>::run([&](auto ic) {
                        constexpr int l = decltype(ic)::value;
                        packed[l] = __byte_perm(packed[l], residue_byte<l>(X, xlo), sel);
                    });
                }
                const int kk = P.k0 + k0;
                uint8_t *dst0 = pbase + image_offset(P.r0 + r, P.tr, nkb, kk / kKB, 0, L, kk % kKB);
#pragma unroll
                for (int l = 0; l < L; l++) *reinterpret_cast<uint32_t *>(dst0 + l * lstride) = packed[l];
            }
        }
    }
}

// ---------------------------------------------------------------- tcgen05 helpers

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

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
// Bounded wait for the phase with the given parity: false when it has not
// completed within limit_ns of wall time (try_wait itself may suspend the
// thread, so the bound is on time, not on iterations) or when another role
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
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(dst), "l"(src), "r"(bytes), "r"(bar) : "memory");
}
// K-major shared-memory descriptor without swizzle (8-row x 16-byte core
// matrices; k halves 128 bytes apart, 8-row groups 256 bytes apart).
__device__ __forceinline__ uint64_t smem_desc_kmajor(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)(128 >> 4) << 16;
    d |= (uint64_t)(256 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}
// kind::i8: S32 accumulator, signed INT8 A and B, K-major, M = 128, N = nt.
__device__ __forceinline__ uint32_t instr_desc_i8(int nt) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(nt >> 3) << 17) | ((uint32_t)(kXRows >> 4) << 24);
}
__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
    asm volatile("{ .reg .pred p; setp.ne.b32 p, %4, 0;\n"
                 "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p; }"
                 :: "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate) : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t *v) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                   "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                   "=r"(v[14]), "=r"(v[15])
                 : "r"(taddr) : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// ---------------------------------------------------------------- modular products

template<int KB>
__global__ void __launch_bounds__(kGemmThreads, 1)
crt_gemm_kernel(const DCrtPanel *__restrict__ panels, const uint8_t *__restrict__ res,
                const DCrtTask *__restrict__ tasks, const DCrtItem *__restrict__ items,
                const int32_t *__restrict__ cta_items, uint8_t *__restrict__ out, const CrtParams cp,
                int32_t stages, int32_t *err, uint64_t wait_ns) {
    // this CTA's items: cta_items[j], j in [cta_items[b], cta_items[b + 1])
    // (every role walks the same list)
    const int j0 = cta_items[blockIdx.x], j1 = cta_items[blockIdx.x + 1];
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    __shared__ __align__(8) uint64_t full_bar[kMaxStages], empty_bar[kMaxStages], accf_bar[2], acce_bar[2], drain_bar;
    __shared__ uint32_t tmem_base_s;
    __shared__ volatile int abort_s;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int L = cp.L;
    if (threadIdx.x == 0) {
        for (int i = 0; i < stages; i++) { mbar_init(&full_bar[i], 1); mbar_init(&empty_bar[i], 1); }
        for (int b = 0; b < 2; b++) { mbar_init(&accf_bar[b], 1); mbar_init(&acce_bar[b], kEpiWarps); }
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

    if (warp == kEpiWarps) {
        // ------------------------------------------------ bulk-copy producer
        if (lane == 0) {
            int st = 0;
            uint32_t ph = 0;
            bool ok = true;
            int armed[kMaxStages];
            for (int i = 0; i < kMaxStages; i++) armed[i] = -1;
            for (int j = j0; j < j1 && ok; j++) {
                const int it = cta_items[j];
                const DCrtItem item = items[it];
                const uint32_t ybytes = (uint32_t)item.nt * kKB;
                for (int l = 0; l < L && ok; l++) {
                    for (int ti = item.t_begin; ti < item.t_end && ok; ti++) {
                        const DCrtTask t = tasks[ti];
                        const int nkb = t.nkb;
                        const int64_t xt = (int64_t)nkb * L * kXTile;          // one M tile's images
                        const uint8_t *ga = res + t.xres + (int64_t)(item.x0 / kXRows) * xt;
                        const uint8_t *gb = res + t.yres + (int64_t)(item.y0 / item.nt) * nkb * L * ybytes;
                        for (int kb = 0; kb < nkb; kb += KB) {
                            if (!mbar_wait(&empty_bar[st], ph ^ 1, &abort_s, wait_ns)) { ok = false; break; }
                            const int nsub = min(KB, nkb - kb);
                            const uint32_t fb = smem_u32(&full_bar[st]);
                            mbar_expect_tx(&full_bar[st], (uint32_t)nsub * ((uint32_t)(item.nx * kXTile) + ybytes));
                            // the stage's k blocks of modulus l: one copy per tile
                            const uint32_t sa = smem0 + st * (KB * kSubBytes);
                            const int64_t img = (int64_t)l * nkb + kb;
                            bulk_load(sa, ga + img * kXTile, (uint32_t)nsub * kXTile, fb);
                            if (item.nx == 2)
                                bulk_load(sa + KB * kXTile, ga + xt + img * kXTile, (uint32_t)nsub * kXTile, fb);
                            bulk_load(sa + 2 * KB * kXTile, gb + img * ybytes, (uint32_t)nsub * ybytes, fb);
                            armed[st] = (int)ph;
                            if (++st == stages) { st = 0; ph ^= 1; }
                        }
                    }
                }
            }
            if (!ok) {
                abort_s = 1;
                atomicExch(err, 7);
            }
            // Every issued copy has landed before the CTA leaves (after an
            // abort the MMA warp no longer consumes them); in a normal run
            // each stage's last phase has completed already.
            volatile int never = 0;
            for (int i = 0; i < stages; i++)
                if (armed[i] >= 0) (void)mbar_wait(&full_bar[i], (uint32_t)armed[i], &never, kWaitNs);
        }
    } else if (warp == kEpiWarps + 1) {
        // ------------------------------------------------ MMA issuer
        if (lane == 0) {
            int st = 0;
            uint32_t ph = 0;
            uint32_t uses[2] = {0, 0};               // fills of each accumulator slot so far
            int rr = 0;                              // slot of the next one-tile fill
            bool ok = true;
            for (int j = j0; j < j1 && ok; j++) {
                const int it = cta_items[j];
                const DCrtItem item = items[it];
                const uint32_t idesc = instr_desc_i8(item.nt);
                for (int l = 0; l < L && ok; l++) {
                    // a two-tile fill takes both slots, a one-tile fill slot rr
                    const int s0 = item.nx == 2 ? 0 : rr;
                    // the epilogue has read the slots' previous fills
                    if (uses[s0] > 0 && !mbar_wait(&acce_bar[s0], (uses[s0] - 1) & 1, &abort_s, wait_ns)) { ok = false; break; }
                    if (item.nx == 2 && uses[1] > 0 && !mbar_wait(&acce_bar[1], (uses[1] - 1) & 1, &abort_s, wait_ns)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t d0 = tmem + (uint32_t)(s0 * kMaxNt);
                    uint32_t acc = 0;
                    for (int ti = item.t_begin; ti < item.t_end && ok; ti++) {
                        const int nkb = tasks[ti].nkb;
                        for (int kb = 0; kb < nkb; kb += KB) {
                            if (!mbar_wait(&full_bar[st], ph, &abort_s, wait_ns)) { ok = false; break; }
                            tc_fence_after();
                            const int nsub = min(KB, nkb - kb);
                            // stage layout: [first M tile's k blocks][second's][N tile's]
                            const uint32_t sbase = smem0 + st * (KB * kSubBytes);
                            const uint32_t ybytes = (uint32_t)item.nt * kKB;
                            for (int j = 0; j < nsub; j++) {
                                const uint32_t a0 = sbase + j * kXTile;
                                const uint64_t db = smem_desc_kmajor(sbase + 2 * KB * kXTile + j * ybytes);
                                umma_i8(d0, smem_desc_kmajor(a0), db, idesc, acc);
                                if (item.nx == 2)
                                    umma_i8(tmem + kMaxNt, smem_desc_kmajor(a0 + KB * kXTile), db, idesc, acc);
                                acc = 1;
                            }
                            umma_commit(&empty_bar[st]);
                            if (++st == stages) { st = 0; ph ^= 1; }
                        }
                    }
                    if (!ok) break;
                    umma_commit(&accf_bar[s0]);
                    uses[s0]++;
                    if (item.nx == 2) { umma_commit(&accf_bar[1]); uses[1]++; }
                    else rr ^= 1;
                }
            }
            if (!ok) {
                abort_s = 1;
                atomicExch(err, 7);
                volatile int never = 0;
                umma_commit(&drain_bar);
                (void)mbar_wait(&drain_bar, 0, &never, kWaitNs);
            }
        }
    } else {
        // ------------------------------------------------ epilogue (warps 0-7)
        // warp w reads TMEM lanes 32 (w % 4) .. + 31 (the lane quarter a warp
        // may access) and every other 16-column chunk, starting at 16 (w / 4)
        const int quarter = warp & 3, chunk0 = (warp >> 2) * 16;
        const int row = quarter * 32 + lane;                      // TMEM lane == tile row
        uint32_t uses[2] = {0, 0};                                // same slot sequence as the MMA warp
        int rr = 0;
        bool ok = true;
        for (int j = j0; j < j1 && ok; j++) {
            const int it = cta_items[j];
            const DCrtItem item = items[it];
            for (int l = 0; l < L; l++) {
                const int s0 = item.nx == 2 ? 0 : rr;
                ok = __all_sync(0xffffffffu, mbar_wait(&accf_bar[s0], uses[s0] & 1, &abort_s, wait_ns));
                if (ok && item.nx == 2) ok = __all_sync(0xffffffffu, mbar_wait(&accf_bar[1], uses[1] & 1, &abort_s, wait_ns));
                if (!ok) break;
                tc_fence_after();
                const double minv = cp.minv_d[l];
                const int mi = cp.m[l];
                for (int xh = 0; xh < item.nx; xh++) {
                    const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)((s0 + xh) * kMaxNt);
                    uint8_t *orow = out + item.res_off + ((int64_t)(l * item.nx + xh) * kXRows + row) * item.nt;
                    for (int c0 = chunk0; c0 < item.nt; c0 += 32) {
                        uint32_t v[16];
                        tmem_ld16(taddr + (uint32_t)c0, v);
                        tmem_wait_ld();
                        uint32_t w[16];
#pragma unroll
                        for (int j = 0; j < 16; j++) {
                            // int32 -> double by bits (2^52 * 1.5 + 2^31 + v, exact); the
                            // quotient q = rint(v / m) is exact (|v| < 2^31), so
                            // r = v - q m lies in [-(m-1)/2, (m-1)/2] (or +-128 for m = 256)
                            const double x = __hiloint2double(0x43380000, (int)(v[j] ^ 0x80000000u)) -
                                             6755401588539392.0;
                            const int q = __double2loint(fma(x, minv, kMagicD));
                            const int r = (int)v[j] - q * mi;
                            w[j] = (uint32_t)(r + ((r >> 31) & mi));           // [0, m)
                        }
                        *reinterpret_cast<uint4 *>(orow + c0) =
                            make_uint4(pack4(w[0], w[1], w[2], w[3]), pack4(w[4], w[5], w[6], w[7]),
                                       pack4(w[8], w[9], w[10], w[11]), pack4(w[12], w[13], w[14], w[15]));
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&acce_bar[s0]);
                    if (item.nx == 2) mbar_arrive(&acce_bar[1]);
                }
                uses[s0]++;
                if (item.nx == 2) uses[1]++;
                else rr ^= 1;
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

// ---------------------------------------------------------------- recombination

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" :: "r"(smem_u32(smem)), "l"(gmem) : "memory");
}

constexpr int kCombCols = 16;                       // tile columns staged per pass

// Units (work item, 128-row half, 16-column chunk): the residues of the
// unit staged in shared memory together with, per tile row and column, its
// exponent and its part of the C offset (one C block: the offsets of its row
// and column; grouped products: the block and coordinates, combined with the
// C block's strides per element); then one thread per element runs Garner
// and writes C.
// SCATTER: each element goes, by atomic adds into a zeroed result, to its C
// block's destinations instead -- blocks of another tensor with their own
// index mappings and coefficients (the terms of a symmetrizer over the
// contraction): dests[drange[cblk]] for a C block of its own (their row and
// column offsets staged like soff), gdcells[gdrange[cell]] with gdcoef for
// a cell of a grouped product.
template<int L, bool SCATTER>
__global__ void __launch_bounds__(256)
crt_combine_kernel(const DCrtPanel *__restrict__ panels, const DCrtItem *__restrict__ items, int32_t nitems,
                   const DCBlock *__restrict__ cblks, const DCrtComp *__restrict__ comps,
                   const int32_t *__restrict__ ctab, const DCrtCell *__restrict__ cells,
                   const uint8_t *__restrict__ out, const int32_t *__restrict__ gidx,
                   const int32_t *__restrict__ ex, const int32_t *__restrict__ ey,
                   const int32_t *__restrict__ ext, const int32_t *__restrict__ eyt, double *__restrict__ C,
                   int32_t add, double scale, const CrtParams cp, const int2 *__restrict__ drange,
                   const DCBlock *__restrict__ dests, const int2 *__restrict__ gdrange,
                   const DCrtCell *__restrict__ gdcells, const double *__restrict__ gdcoef) {
    constexpr int kTab = kXRows + kCombCols;
    __shared__ __align__(16) uint8_t sres[L][kXRows][kCombCols];
    __shared__ int64_t sdoff[SCATTER ? kCrtMaxDests * kTab : 1];  // SCATTER: each destination's offsets
    __shared__ int64_t soff[kXRows + kCombCols];               // one C block: row / column offsets
    __shared__ int32_t sexp[kXRows + kCombCols];               // exponents of tile rows / columns
    __shared__ int32_t sco[kXRows + kCombCols][1 + kCrtSideDims];   // grouped: block, coordinates
    for (int u = blockIdx.x; u < nitems * 32; u += gridDim.x) {
        const DCrtItem item = items[u >> 5];
        const int xh = (u >> 4) & 1, c0 = (u & 15) * kCombCols;
        const DCrtComp *cc = item.comp >= 0 ? &comps[item.comp] : nullptr;
        const DCBlock *cb1 = cc ? nullptr : &cblks[item.cblk];
        const int rows = cc ? cc->rows : cb1->M, cols = cc ? cc->cols : cb1->N;
        const int xext = cp.swap ? cols : rows, yext = cp.swap ? rows : cols;
        const int yc = min(item.nt, yext - item.y0);
        if (xh >= item.nx || c0 >= yc) continue;                     // uniform over the CTA
        const int xb = item.x0 + xh * kXRows;                        // first row of this half
        const int xr = min(kXRows, xext - xb);
        int d0 = 0, nd = 0;                                          // SCATTER: the C block's destinations
        if constexpr (SCATTER) {
            if (!cc) {
                const int2 dr = drange[item.cblk];
                d0 = dr.x;
                nd = min(dr.y - dr.x, kCrtMaxDests);
            }
        }
        __syncthreads();                                             // the previous unit is done
        for (int i = threadIdx.x; i < L * kXRows; i += blockDim.x) {
            const int l = i / kXRows, r = i - l * kXRows;
            cp_async16(&sres[l][r][0], out + item.res_off + ((int64_t)(l * item.nx + xh) * kXRows + r) * item.nt + c0);
        }
        for (int i = threadIdx.x; i < kXRows + kCombCols; i += blockDim.x) {
            const bool isx = i < kXRows;
            const int j = isx ? i : i - kXRows;
            if (isx ? j >= xr : c0 + j >= yc) continue;
            const int idx = isx ? xb + j : item.y0 + c0 + j;           // tile row / column
            // the exponent the residues were formed with: the bound, or the
            // exact exponent of a row the residue pass redid
            const int g = isx ? gidx[panels[item.gx].g_off + idx] : gidx[panels[item.gy].g_off + idx];
            sexp[i] = isx ? max(ex[g], ext[g]) : max(ey[g], eyt[g]);
            const bool crow = isx != (cp.swap != 0);                  // a row of C (side of A)
            if (cc) {
                const int32_t *e = ctab + (crow ? cc->row_off : cc->col_off) + (1 + kCrtSideDims) * idx;
#pragma unroll
                for (int k = 0; k <= kCrtSideDims; k++) sco[i][k] = e[k];
            } else {
                soff[i] = crow ? mixed_offset(idx, cb1->nm, cb1->mext, cb1->mc_str)
                               : mixed_offset(idx, cb1->nn, cb1->next, cb1->nc_str);
                if constexpr (SCATTER)
                    for (int d = 0; d < nd; d++) {
                        const DCBlock &db = dests[d0 + d];
                        sdoff[d * kTab + i] = crow ? mixed_offset(idx, db.nm, db.mext, db.mc_str)
                                                   : mixed_offset(idx, db.nn, db.next, db.nc_str);
                    }
            }
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        __syncthreads();
        for (int e = threadIdx.x; e < kXRows * kCombCols; e += blockDim.x) {
            int r, c;
            if (cp.swap) { r = e & (kXRows - 1); c = e >> 7; }      // C rows along the tile columns
            else { c = e & (kCombCols - 1); r = e >> 4; }
            if (r >= xr || c0 + c >= yc) continue;
            int64_t off = 0;
            int cell = -1;
            const int32_t *cm = nullptr, *cn = nullptr;
            if (cc) {                                                // grouped: the C block of (r, c)
                const int32_t *cx = sco[r], *cy = sco[kXRows + c];
                cm = cp.swap ? cy : cx;
                cn = cp.swap ? cx : cy;
                cell = ctab[cc->cell_off + cm[0] * cc->ncb + cn[0]];
                if (cell < 0) continue;
                if constexpr (!SCATTER) {
                    const DCrtCell &cl = cells[cell];
                    off = cl.c_off;
#pragma unroll
                    for (int k = 0; k < kCrtSideDims; k++) off += (int64_t)cm[1 + k] * cl.ms[k] + (int64_t)cn[1 + k] * cl.ns[k];
                }
            } else if constexpr (!SCATTER) {
                off = cb1->c_off + soff[r] + soff[kXRows + c];
            }
            // Garner: balanced mixed-radix digits v_i of the residues.  Every
            // quantity is an integer below 2^19 in magnitude (|r_i D| <=
            // 255 * 128, |v_j D| <= 128 * 128, at most 15 terms), so FP32
            // holds it exactly; the quotient rint(t / m_i) from one FMA is
            // exact for odd m_i (t / m_i stays 1/(2 m_i) away from a half
            // integer, far above the product's rounding), which leaves t
            // in [-(m_i - 1)/2, (m_i - 1)/2].
            float v[L];
            StaticFor<0, L>::run([&](auto ii) {
                constexpr int i = decltype(ii)::value;
                const float ri = __int_as_float(0x4B000000 | (int)sres[i][r][c]) - 8388608.0f;
                if constexpr (i == 0) {
                    v[0] = ri >= 128.0f ? ri - 256.0f : ri;             // m_0 = 256: the byte itself
                } else {
                    constexpr float mi = (float)crt_modulus(i), minv = 1.0f / (float)crt_modulus(i);
                    float t = ri * (float)crt_garner_d(0, i);
                    StaticFor<0, i>::run([&](auto jj) {
                        constexpr int j = decltype(jj)::value;
                        t = fmaf(-v[j], (float)crt_garner_d(j, i), t);
                    });
                    v[i] = fmaf(-(fmaf(t, minv, kMagicF) - kMagicF), mi, t);
                }
            });
            // digits to double by bits (|v| < 2^22): float 1.5*2^23 + v -> int -> double
            auto digit = [](float f) {
                const int iv = __float_as_int(f + kMagicF) - 0x4B400000;
                return __hiloint2double(0x43380000, iv ^ (int)0x80000000) - 6755401588539392.0;
            };
            double X = digit(v[L - 1]);
#pragma unroll
            for (int i = L - 2; i >= 0; i--) X = fma(X, (double)crt_modulus(i), digit(v[i]));
            // 2^(e_row + e_col - 2P) from its bits (a row without exponent has X = 0)
            const int e2 = sexp[r] + sexp[kXRows + c] - 2 * cp.P;
            const double p2 = e2 < -1022 ? 0.0 : __hiloint2double((min(e2, 1023) + 1023) << 20, 0);
            const double val = scale * (X * p2);
            if constexpr (SCATTER) {
                if (cc) {
                    const int2 dr = gdrange[cell];
                    for (int d = dr.x; d < dr.y; d++) {
                        const DCrtCell &dl = gdcells[d];
                        int64_t o = dl.c_off;
#pragma unroll
                        for (int k = 0; k < kCrtSideDims; k++) o += (int64_t)cm[1 + k] * dl.ms[k] + (int64_t)cn[1 + k] * dl.ns[k];
                        atomicAdd(C + o, gdcoef[d] * val);
                    }
                } else {
                    for (int d = 0; d < nd; d++)
                        atomicAdd(C + dests[d0 + d].c_off + sdoff[d * kTab + r] + sdoff[d * kTab + kXRows + c],
                                  dests[d0 + d].scale * val);
                }
            } else {
                double *dst = C + off;
                if (add) *dst += val;
                else *dst = val;
            }
        }
    }
}

int g_crt_nsm = 0;

int num_sms() {
    if (g_crt_nsm == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_crt_nsm, cudaDevAttrMultiProcessorCount, dev);
    }
    return g_crt_nsm;
}

}  // namespace

cudaError_t launch_crt_exponents(const DCrtPanel *panels, const int4 *units, int32_t nunits, int32_t nx,
                                 int32_t ny, const double *a, const double *b, const int32_t *gidx, int32_t *ex,
                                 int32_t *ey, int32_t sample, cudaStream_t s) {
    if (nunits <= 0) return cudaSuccess;
    const int grid = nunits;                               // one unit per CTA
    crt_exp_kernel<<<grid, kSplitThreads, 0, s>>>(panels, units, nunits, a, b, gidx, ex, ey, sample);
    return cudaGetLastError();
}

cudaError_t launch_crt_fill(int32_t nx, int32_t ny, int32_t *ex, int32_t *ey, cudaStream_t s) {
    crt_fill_kernel<<<64, 256, 0, s>>>(ex, nx, kNoExp);
    crt_fill_kernel<<<64, 256, 0, s>>>(ey, ny, kNoExp);
    return cudaGetLastError();
}

bool crt_unit_sampled(const DCrtPanel &p, int unit_map) { return sampled_panel(p, unit_map); }
int64_t crt_sampled_elems(const DCrtPanel &p) {
    // elements the sampled exponent pass reads of one row
    const int64_t runs = ((int64_t)p.K + 32 * kSampleGroups - 1) / (32 * kSampleGroups);
    return std::min<int64_t>(32 * runs, p.K);
}

template<int L, class FC>
cudaError_t launch_fused_l(const DCrtPanel *panels, const DCrtFamily *fams, const int32_t *famp,
                           const int32_t *famt, const int4 *units, int32_t nunits, const double *a,
                           const double *b, const int32_t *gidx, int32_t *ex, int32_t *ey, uint8_t *res,
                           const CrtParams &cp, cudaStream_t s) {
    const int maxg = FC::kCtasPerSm * num_sms();
    const int grid = nunits < maxg ? nunits : maxg;
    crt_fused_kernel<L, FC><<<grid, FC::kThreads, 0, s>>>(panels, fams, famp, famt, units, nunits, a, b, gidx, ex,
                                                          ey, res, cp);
    return cudaGetLastError();
}

template<class FC>
cudaError_t launch_fused_cfg(const DCrtPanel *panels, const DCrtFamily *fams, const int32_t *famp,
                             const int32_t *famt, const int4 *units, int32_t nunits, const double *a,
                             const double *b, const int32_t *gidx, int32_t *ex, int32_t *ey, uint8_t *res,
                             const CrtParams &cp, cudaStream_t s) {
    switch (cp.L) {
#define CASE_L(n) case n: return launch_fused_l<n, FC>(panels, fams, famp, famt, units, nunits, a, b, gidx, ex, ey, res, cp, s);
    CASE_L(8) CASE_L(9) CASE_L(10) CASE_L(11) CASE_L(12) CASE_L(13) CASE_L(14) CASE_L(15) CASE_L(16)
#undef CASE_L
    default: return cudaErrorInvalidValue;
    }
}

int crt_fuse_rows(int shape) { return shape == 1 || shape == 2 ? 2 : 0; }

cudaError_t launch_crt_fused(int shape, const DCrtPanel *panels, const DCrtFamily *fams, const int32_t *famp,
                             const int32_t *famt, const int4 *units, int32_t nunits, const double *a,
                             const double *b, const int32_t *gidx, int32_t *ex, int32_t *ey, uint8_t *res,
                             const CrtParams &cp, cudaStream_t s) {
    if (nunits <= 0) return cudaSuccess;
    // 1: 2 rows, 512 threads, 2 CTAs/SM; 2: 2 rows, 256 threads, 4/SM.
    // (1-row units, whose residue stores fill half sectors, ran 3.5x slower
    // than these; 4-row units with 2 CTAs/SM 20 % slower.)
    switch (shape) {
    case 1: return launch_fused_cfg<FuseCfg<2, 512, 2>>(panels, fams, famp, famt, units, nunits, a, b, gidx, ex, ey, res, cp, s);
    case 2: return launch_fused_cfg<FuseCfg<2, 256, 4>>(panels, fams, famp, famt, units, nunits, a, b, gidx, ex, ey, res, cp, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_crt_residues(const DCrtPanel *panels, const int4 *units, int32_t nunits,
                                const double *a, const double *b, const int32_t *gidx, const int32_t *ex,
                                const int32_t *ey, int32_t *ext, int32_t *eyt, int32_t sample, int32_t redo,
                                uint8_t *res, const CrtParams &cp, cudaStream_t s) {
    if (nunits <= 0) return cudaSuccess;
    const int grid = nunits;                               // one unit per CTA
    switch (cp.L) {
#define CASE_L(n) case n: crt_res_kernel<n><<<grid, kSplitThreads, 0, s>>>(panels, units, nunits, a, b, gidx, ex, ey, ext, eyt, sample, redo, res, cp); break;
    CASE_L(8) CASE_L(9) CASE_L(10) CASE_L(11) CASE_L(12) CASE_L(13) CASE_L(14) CASE_L(15) CASE_L(16)
#undef CASE_L
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template<int KB>
cudaError_t launch_gemm_kb(const DCrtPanel *panels, const uint8_t *res, const DCrtTask *tasks,
                           const DCrtItem *items, const int32_t *cta_items, int32_t ncta, uint8_t *out, const CrtParams &cp,
                           int32_t *err, uint64_t wait_ns, cudaStream_t s) {
    constexpr int stage_bytes = KB * kSubBytes;
    int stages = (200 * 1024) / stage_bytes;
    if (stages > kMaxStages) stages = kMaxStages;
    const size_t smem = (size_t)stages * stage_bytes + 1024;
    cudaError_t e = cudaFuncSetAttribute(crt_gemm_kernel<KB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    crt_gemm_kernel<KB><<<ncta, kGemmThreads, smem, s>>>(panels, res, tasks, items, cta_items, out, cp, stages, err,
                                                         wait_ns);
    return cudaGetLastError();
}

cudaError_t launch_crt_gemm(const DCrtPanel *panels, const uint8_t *res, const DCrtTask *tasks,
                            const DCrtItem *items, const int32_t *cta_items, int32_t ncta, uint8_t *out, const CrtParams &cp,
                            int32_t *err, uint64_t wait_ns, int32_t stage_kb, cudaStream_t s) {
    if (ncta <= 0) return cudaSuccess;
    // k blocks per pipeline stage: 2 (6 stages of 32 KB), 3 (4 x 48 KB), 4
    // (3 x 64 KB, the default), 6 (2 x 96 KB)
    switch (stage_kb) {
    case 2: return launch_gemm_kb<2>(panels, res, tasks, items, cta_items, ncta, out, cp, err, wait_ns, s);
    case 3: return launch_gemm_kb<3>(panels, res, tasks, items, cta_items, ncta, out, cp, err, wait_ns, s);
    case 6: return launch_gemm_kb<6>(panels, res, tasks, items, cta_items, ncta, out, cp, err, wait_ns, s);
    default: return launch_gemm_kb<4>(panels, res, tasks, items, cta_items, ncta, out, cp, err, wait_ns, s);
    }
}

// Resident CTAs per SM of a recombination instantiation (its registers and
// shared memory), found once.
template<int L, bool SCATTER>
int combine_ctas_per_sm() {
    static const int v = [] {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, crt_combine_kernel<L, SCATTER>, 256, 0) != cudaSuccess ||
            n < 1)
            n = 1;
        return n;
    }();
    return v;
}

cudaError_t launch_crt_combine(const DCrtPanel *panels, const DCrtItem *items, int32_t nitems,
                               const DCBlock *cblks, const DCrtComp *comps, const int32_t *ctab,
                               const DCrtCell *cells, const uint8_t *out, const int32_t *gidx,
                               const int32_t *ex, const int32_t *ey, const int32_t *ext, const int32_t *eyt, double *c, int32_t add, double scale,
                               const CrtParams &cp, cudaStream_t s, const CrtDests *dd) {
    if (nitems <= 0) return cudaSuccess;
    // 8 CTAs per SM (6 resident) striding over the units; with fewer than 16
    // units per CTA the partial second wave of that grid sets the time, and
    // one wave of resident CTAs is used instead
    const int units = 32 * nitems;
    auto grid_of = [&](int resident) {
        const int g = units < 16 * 8 * num_sms() ? resident * num_sms() : 8 * num_sms();
        return units < g ? units : g;
    };
    switch (cp.L) {
#define CASE_L(n) case n: \
        if (dd) crt_combine_kernel<n, true><<<grid_of(combine_ctas_per_sm<n, true>()), 256, 0, s>>>(panels, items, nitems, cblks, comps, ctab, cells, out, gidx, ex, ey, ext, eyt, c, 0, scale, cp, dd->drange, dd->dests, dd->gdrange, dd->gdcells, dd->gdcoef); \
        else crt_combine_kernel<n, false><<<grid_of(combine_ctas_per_sm<n, false>()), 256, 0, s>>>(panels, items, nitems, cblks, comps, ctab, cells, out, gidx, ex, ey, ext, eyt, c, add, scale, cp, nullptr, nullptr, nullptr, nullptr, nullptr); \
        break;
    CASE_L(8) CASE_L(9) CASE_L(10) CASE_L(11) CASE_L(12) CASE_L(13) CASE_L(14) CASE_L(15) CASE_L(16)
#undef CASE_L
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace ltg
