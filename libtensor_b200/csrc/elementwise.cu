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
// destination element (+8 when accumulating).  Threads run along the
// innermost destination dimension; when a term reads that dimension with a
// non-unit stride (a transposition such as P(ab)), a shared-memory tile turns
// the strided reads into coalesced ones.
#include "ltg_device.cuh"

namespace ltg {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ int64_t outer_base(int64_t row, int nout, const int32_t *ext,
                                              const int32_t *str) {
    // decompose row over the outer dims (ext[0..nout)) row-major
    int64_t off = 0;
    for (int i = nout - 1; i >= 0; i--) {
        int64_t e = ext[i];
        int64_t q = row / e;
        off += (row - q * e) * str[i];
        row = q;
    }
    return off;
}

// Generic path: threads along the innermost dim (coalesced destination).
__global__ void __launch_bounds__(kThreads)
transfer_kernel(const DJob *__restrict__ jobs, const DTerm *__restrict__ terms,
                const DUnit *__restrict__ units, int32_t nunits,
                const double *const *__restrict__ srcs, double *__restrict__ dst,
                int32_t accumulate, double beta) {
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const DUnit un = units[u];
        const DJob &j = jobs[un.job];
        const int inner = j.inner;
        int tin = kThreads;
        while (tin / 2 >= inner && tin > 1) tin >>= 1;
        const int rows_per_pass = kThreads / tin;
        const int i0 = threadIdx.x % tin;
        for (int64_t r = un.row_begin + threadIdx.x / tin; r < un.row_end; r += rows_per_pass) {
            int64_t sb[kMaxTerms];
            for (int t = 0; t < j.nterms; t++)
                sb[t] = terms[j.term0 + t].src_off +
                        outer_base(r, j.ndim - 1, j.ext, terms[j.term0 + t].sstr);
            double *d = dst + j.dst_off + r * inner;
            for (int i = i0; i < inner; i += tin) {
                double v = 0.0;
                for (int t = 0; t < j.nterms; t++) {
                    const DTerm &tm = terms[j.term0 + t];
                    v += tm.coeff * srcs[tm.src][sb[t] + (int64_t)i * tm.sstr[j.ndim - 1]];
                }
                if (accumulate) d[i] = d[i] + beta * v;
                else d[i] = v;
            }
        }
    }
}

// Dot product: per unit partial sum, then one fixed-order reduction.
__global__ void __launch_bounds__(kThreads)
dot_kernel(const DJob *__restrict__ jobs, const DTerm *__restrict__ terms,
           const DUnit *__restrict__ units, int32_t nunits,
           const double *__restrict__ a, const double *__restrict__ b,
           double *__restrict__ partials) {
    __shared__ double red[kThreads];
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const DUnit un = units[u];
        const DJob &j = jobs[un.job];
        const DTerm &ta = terms[j.term0], &tb = terms[j.term0 + 1];
        const int inner = j.inner;
        int tin = kThreads;
        while (tin / 2 >= inner && tin > 1) tin >>= 1;
        const int rows_per_pass = kThreads / tin;
        const int i0 = threadIdx.x % tin;
        double s = 0.0;
        for (int64_t r = un.row_begin + threadIdx.x / tin; r < un.row_end; r += rows_per_pass) {
            int64_t oa = ta.src_off + outer_base(r, j.ndim - 1, j.ext, ta.sstr);
            int64_t ob = tb.src_off + outer_base(r, j.ndim - 1, j.ext, tb.sstr);
            const int64_t sa = ta.sstr[j.ndim - 1], sbb = tb.sstr[j.ndim - 1];
            for (int i = i0; i < inner; i += tin) s += a[oa + i * sa] * b[ob + i * sbb];
        }
        red[threadIdx.x] = s;
        __syncthreads();
        for (int w = kThreads / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) partials[u] = red[0] * ta.coeff;
        __syncthreads();
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

int grid_for(int64_t units) {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    int64_t g = units < (int64_t)nsm * 8 ? units : (int64_t)nsm * 8;
    return g < 1 ? 1 : (int)g;
}

}  // namespace

cudaError_t launch_transfer(const DJob *jobs, const DTerm *terms, const DUnit *units,
                            int32_t nunits, const double *const *srcs, double *dst,
                            int32_t accumulate, double beta, cudaStream_t s) {
    if (nunits <= 0) return cudaSuccess;
    transfer_kernel<<<grid_for(nunits), kThreads, 0, s>>>(jobs, terms, units, nunits, srcs, dst,
                                                          accumulate, beta);
    return cudaGetLastError();
}

cudaError_t launch_dot(const DJob *jobs, const DTerm *terms, const DUnit *units,
                       int32_t nunits, const double *a, const double *b, double *partials,
                       double *out, cudaStream_t s) {
    if (nunits <= 0) return cudaMemsetAsync(out, 0, sizeof(double), s);
    dot_kernel<<<grid_for(nunits), kThreads, 0, s>>>(jobs, terms, units, nunits, a, b, partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    reduce_kernel<<<1, kThreads, 0, s>>>(partials, nunits, out);
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
