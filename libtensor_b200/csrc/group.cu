// Grouped products of the plain FP64 contraction: data movement around one
// dense DMMA product per group (the grouping itself is planned on the host,
// see crt_groups in ltg_capi.cu).
//  - gather_cells_kernel: every operand cell (a canonical block read through
//    the pair's orbit transform, times its sign) copied into its place in a
//    dense group panel (rows x k, k contiguous), each thread on a fixed k
//    (its offset found once) stepping over rows; non-contiguous k offsets
//    come from a shared-memory table built once per unit;
//  - scatter_groups_kernel: the dense group result (C rows x C columns of the
//    group) written into the C blocks of the grid (assign or add), through
//    the same placement tables as the modular mode's recombination.
// Cells that no pair uses are never written: their panel entries stay zero
// from the buffer's clearing when the plan was built.
#include "ltg_device.cuh"

namespace ltg {
namespace {

constexpr int kGatherThreads = 256;
constexpr int kGatherKoff = 4096;

__device__ __forceinline__ int64_t gmixed(int32_t lin, int n, const int32_t *ext, const int32_t *str) {
    int64_t off = 0;
    for (int i = n - 1; i >= 0; i--) {
        const int32_t e = ext[i];
        const int32_t q = lin / e;
        off += (int64_t)(lin - q * e) * str[i];
        lin = q;
    }
    return off;
}

// Units: (piece, first row, rows, unused).
__global__ void __launch_bounds__(kGatherThreads)
gather_cells_kernel(const DGather *__restrict__ pieces, const int4 *__restrict__ units, int32_t nunits,
                    const double *__restrict__ A, const double *__restrict__ B, double *__restrict__ buf) {
    __shared__ int32_t koff[kGatherKoff];
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const int4 un = units[u];
        const DGather &P = pieces[un.x];
        const bool contig = P.nk == 0 || (P.nk == 1 && P.kstr[0] == 1);
        const bool tab = !contig && P.K <= kGatherKoff;          // uniform over the CTA
        if (tab) {
            __syncthreads();                                      // the previous unit's readers are done
            for (int k = threadIdx.x; k < P.K; k += blockDim.x) koff[k] = (int32_t)gmixed(k, P.nk, P.kext, P.kstr);
            __syncthreads();
        }
        const double *src = (P.src ? B : A) + P.src_off;
        const double coef = (double)P.coef;
        if (P.K <= kGatherThreads) {
            // a fixed k per thread (its offset found once), rows dr apart
            const int dr = kGatherThreads / P.K, r0 = threadIdx.x / P.K, k = threadIdx.x - r0 * P.K;
            if (r0 < dr) {
                const int64_t ko = contig ? k : (tab ? koff[k] : gmixed(k, P.nk, P.kext, P.kstr));
                double *d = buf + P.dst_off + (int64_t)(un.y + r0) * P.ld + k;
                for (int r = un.y + r0; r < un.y + un.z; r += dr, d += (int64_t)dr * P.ld)
                    *d = coef * src[gmixed(r, P.nr, P.rext, P.rstr) + ko];
            }
        } else {
            for (int r = un.y; r < un.y + un.z; r++) {
                const double *row = src + gmixed(r, P.nr, P.rext, P.rstr);
                double *d = buf + P.dst_off + (int64_t)r * P.ld;
                for (int k = threadIdx.x; k < P.K; k += kGatherThreads)
                    d[k] = coef * row[contig ? k : (tab ? koff[k] : gmixed(k, P.nk, P.kext, P.kstr))];
            }
        }
    }
}

// Units: (group, row of the group's result).
__global__ void __launch_bounds__(256)
scatter_groups_kernel(const DCrtComp *__restrict__ comps, const int64_t *__restrict__ res_off,
                      const int32_t *__restrict__ ctab, const DCrtCell *__restrict__ cells,
                      const int2 *__restrict__ units, int32_t nunits, const double *__restrict__ buf,
                      double *__restrict__ C, double scale, int32_t add) {
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const int2 un = units[u];
        const DCrtComp cc = comps[un.x];
        const int m = un.y;
        const int32_t *re = ctab + cc.row_off + (1 + kCrtSideDims) * m;
        const int rb = re[0];
        const double *src = buf + res_off[un.x] + (int64_t)m * cc.cols;
        for (int n = threadIdx.x; n < cc.cols; n += blockDim.x) {
            const int32_t *ce = ctab + cc.col_off + (1 + kCrtSideDims) * n;
            const int cell = ctab[cc.cell_off + rb * cc.ncb + ce[0]];
            if (cell < 0) continue;
            const DCrtCell &cl = cells[cell];
            int64_t off = cl.c_off;
#pragma unroll
            for (int k = 0; k < kCrtSideDims; k++) off += (int64_t)re[1 + k] * cl.ms[k] + (int64_t)ce[1 + k] * cl.ns[k];
            const double v = scale * src[n];
            if (add) C[off] += v;
            else C[off] = v;
        }
    }
}

// The same rows, each element added (atomically, into a zeroed result) to
// the destinations of its cell: dcells[drange[cell].x .. drange[cell].y),
// each a block of another tensor with its own strides, times dcoef (the
// terms of a symmetrizer over the contraction).
__global__ void __launch_bounds__(256)
scatter_groups_dest_kernel(const DCrtComp *__restrict__ comps, const int64_t *__restrict__ res_off,
                           const int32_t *__restrict__ ctab, const int2 *__restrict__ drange,
                           const DCrtCell *__restrict__ dcells, const double *__restrict__ dcoef,
                           const int2 *__restrict__ units, int32_t nunits, const double *__restrict__ buf,
                           double *__restrict__ R, double scale) {
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const int2 un = units[u];
        const DCrtComp cc = comps[un.x];
        const int m = un.y;
        const int32_t *re = ctab + cc.row_off + (1 + kCrtSideDims) * m;
        const int rb = re[0];
        const double *src = buf + res_off[un.x] + (int64_t)m * cc.cols;
        for (int n = threadIdx.x; n < cc.cols; n += blockDim.x) {
            const int32_t *ce = ctab + cc.col_off + (1 + kCrtSideDims) * n;
            const int cell = ctab[cc.cell_off + rb * cc.ncb + ce[0]];
            if (cell < 0) continue;
            const int2 dr = drange[cell];
            const double v = scale * src[n];
            for (int d = dr.x; d < dr.y; d++) {
                const DCrtCell &dl = dcells[d];
                int64_t off = dl.c_off;
#pragma unroll
                for (int k = 0; k < kCrtSideDims; k++) off += (int64_t)re[1 + k] * dl.ms[k] + (int64_t)ce[1 + k] * dl.ns[k];
                atomicAdd(R + off, dcoef[d] * v);
            }
        }
    }
}

int g_group_nsm = 0;

int group_sms() {
    if (g_group_nsm == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_group_nsm, cudaDevAttrMultiProcessorCount, dev);
    }
    return g_group_nsm;
}

// One wave of resident CTAs of a grid-striding kernel (256 threads, no
// dynamic shared memory): more CTAs than fit leave a partial last wave that
// sets the launch's time.
template<class K>
int resident_grid(K kernel) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, 256, 0) != cudaSuccess || n < 1) n = 1;
    return n * group_sms();
}

}  // namespace

cudaError_t launch_gather_cells(const DGather *pieces, const int4 *units, int32_t nunits, const double *a,
                                const double *b, double *buf, cudaStream_t s) {
    if (nunits <= 0) return cudaSuccess;
    static const int resident = resident_grid(gather_cells_kernel);
    const int grid = nunits < resident ? nunits : resident;
    gather_cells_kernel<<<grid, kGatherThreads, 0, s>>>(pieces, units, nunits, a, b, buf);
    return cudaGetLastError();
}

cudaError_t launch_scatter_groups(const DCrtComp *comps, const int64_t *res_off, const int32_t *ctab,
                                  const DCrtCell *cells, const int2 *units, int32_t nunits, const double *buf,
                                  double *c, double scale, int32_t add, cudaStream_t s) {
    if (nunits <= 0) return cudaSuccess;
    static const int resident = resident_grid(scatter_groups_kernel);
    const int grid = nunits < resident ? nunits : resident;
    scatter_groups_kernel<<<grid, 256, 0, s>>>(comps, res_off, ctab, cells, units, nunits, buf, c, scale, add);
    return cudaGetLastError();
}

cudaError_t launch_scatter_groups_dest(const DCrtComp *comps, const int64_t *res_off, const int32_t *ctab,
                                       const int2 *drange, const DCrtCell *dcells, const double *dcoef,
                                       const int2 *units, int32_t nunits, const double *buf, double *r,
                                       double scale, cudaStream_t s) {
    if (nunits <= 0) return cudaSuccess;
    static const int resident = resident_grid(scatter_groups_dest_kernel);
    const int grid = nunits < resident ? nunits : resident;
    scatter_groups_dest_kernel<<<grid, 256, 0, s>>>(comps, res_off, ctab, drange, dcells, dcoef, units, nunits, buf,
                                                    r, scale);
    return cudaGetLastError();
}

}  // namespace ltg
