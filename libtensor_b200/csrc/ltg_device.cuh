// Device-side data layouts of the B200 block-tensor path and the kernel
// launchers shared by the C ABI layer.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ltg {

constexpr int kDevMaxSub = 4;     // sub-dimension groups per GEMM axis
constexpr int kDevMaxOrder = 8;

// ---------------------------------------------------------------- contraction

// One (C block, pair) product:  C[m,n] += coeff * sum_k A[m,k] * B[n,k]
// with A/B element offsets  a_off + sum_i digit_m[i]*ma_str[i] + sum_j digit_k[j]*ka_str[j].
// All within-block strides fit 32 bits (a block holds < 2^31 elements).
struct DTask {
    int64_t a_off, b_off;
    double coeff;                 // relative to the owning C block's scale
    int32_t K;
    int32_t nk, nm, nn;
    int32_t kext[kDevMaxSub], ka_str[kDevMaxSub], kb_str[kDevMaxSub];
    int32_t mext[kDevMaxSub], ma_str[kDevMaxSub];
    int32_t next[kDevMaxSub], nb_str[kDevMaxSub];
    int32_t vec_a, vec_b;         // 16-byte loads allowed (contiguous, even-aligned k pairs)
};

// One canonical C block of the schedule.
struct DCBlock {
    int64_t c_off;
    double scale;                 // kc (and d in add mode) times the first pair's coefficient
    int32_t M, N;
    int32_t nm, nn;
    int32_t mext[kDevMaxSub], mc_str[kDevMaxSub];
    int32_t next[kDevMaxSub], nc_str[kDevMaxSub];
    int32_t t_begin, t_end;       // task range
};

// One CTA work item: an (m, n) tile of a C block, over the k tiles
// [kt0, kt1) of the C block's task sequence (every task's k tiles in task
// order).  slot < 0: the item covers all k tiles and writes C itself;
// slot >= 0: a k chunk whose partial tile goes to workspace slot `slot`,
// summed in chunk order by the split reduction.
struct DItem {
    int32_t cblk;
    int32_t m0, n0;
    int32_t slot;
    int32_t kt0, kt1;
};

// A tile whose k range was split into nparts chunks (workspace slots
// slot0 .. slot0 + nparts - 1, in k order).
struct DSplit {
    int32_t cblk;
    int32_t m0, n0;
    int32_t nparts;
    int32_t slot0;
    int32_t pad;
};

inline DItem make_item(int32_t cblk, int32_t m0, int32_t n0) {
    DItem it;
    it.cblk = cblk; it.m0 = m0; it.n0 = n0;
    it.slot = -1; it.kt0 = 0; it.kt1 = INT32_MAX;
    return it;
}

// ---------------------------------------------------------------- split precision

// Slice element kinds of the split-precision contraction.
enum OzKind { kOzInt8 = 0, kOzBf16 = 1, kOzE4m3 = 2 };

// One split operand panel: the matricised view (rows x K) of a canonical
// block, cut into S integer-valued slices stored as shared-memory tile images
// (per row tile, 32-byte k block and slice), rows padded to 128 and K to 32
// elements.
struct DPanel {
    int64_t src_off;              // FP64 source block offset (elements)
    int64_t slice_off;            // byte offset of slice 0 in the slice arena
    int32_t exp_off;              // first row exponent in the exponent arena
    int32_t src;                  // 0: A arena, 1: B arena
    int32_t rows, K, rows_pad, K_pad;
    int32_t nr, nk;
    int32_t rext[kDevMaxSub], rstr[kDevMaxSub];
    int32_t kext[kDevMaxSub], kstr[kDevMaxSub];
};

struct DOzTask {
    int32_t pa, pb;               // panels of A and B
    double coeff;                 // relative coefficient of the pair
};

// ---------------------------------------------------------------- CRT (modular) split precision

constexpr int kCrtMaxModuli = 16;

// One operand panel of the modular contraction: the matricised view (rows x K)
// of a canonical block, with the pair's integer coefficient folded in, scaled
// row by row to integers and stored as its residues modulo each modulus, in
// shared-memory tile images (per tile of tr rows, modulus, 32-byte k block).
struct DCrtPanel {
    int64_t src_off;              // FP64 source block offset (elements)
    int64_t res_off;              // byte offset of the tile images
    int32_t src;                  // 0: A arena, 1: B arena
    int32_t side;                 // 0: MMA M operand (128-row tiles), 1: MMA N operand
    int32_t rows, K, rows_pad, K_pad;
    int32_t tr;                   // rows per tile image (128, or the N tile width)
    int32_t coef;                 // integer coefficient folded into the residues
    int32_t g_off;                // first of this panel's rows in the global row-index array
    int32_t nr, nk;
    int32_t rext[kDevMaxSub], rstr[kDevMaxSub];
    int32_t kext[kDevMaxSub], kstr[kDevMaxSub];
    // Placement in the tile images: rows [r0, r0 + wrows) and k [k0, k0 + wk)
    // are written (the padding included; k0 and wk multiples of 4).  A panel
    // of its own has r0 = k0 = 0, wrows = rows_pad, wk = K_pad; a piece of a
    // grouped panel writes its cell of the group's images, whose geometry
    // (tr, K_pad) it carries.
    int32_t r0, k0, wrows, wk;
};

// A row family of the modular split: panels whose rows feed the same global
// rows of C, row r of every panel the same global row, and nothing else
// feeds those rows (so a row's exponent is the maximum over the family's
// rows r alone).  Panels famp[p_begin .. p_end); famt[q] = first 16-wide k
// tile of panel famp[q] in the family's tile sequence (famt[p_end] = ntiles).
struct DCrtFamily {
    int32_t p_begin, p_end;
    int32_t rows;
    int32_t ntiles;
};

struct DCrtTask {
    int32_t px, py;               // MMA M-side and N-side panels of one pair
    int64_t xres, yres;           // byte offsets of their tile images
    int32_t nkb;                  // 32-byte k blocks
    int32_t pad;
};

// One CTA work item: an (nx * 128) x nt tile of one C block (in MMA
// orientation: rows from the M-side operand, columns from the N-side
// operand); the nx <= 2 row tiles share every N-side operand tile.
struct DCrtItem {
    int32_t cblk;
    int32_t x0, y0;               // first M-side row, first N-side row
    int32_t nt;                   // N tile width (multiple of 16, <= 256)
    int32_t nx;                   // 128-row tiles (1 or 2)
    int32_t t_begin, t_end;       // pairs (DCrtTask range)
    int32_t gx, gy;               // panels whose global row indices label the tile
    int32_t comp;                 // grouped product (DCrtComp) or -1 for one C block (cblk)
    int64_t res_off;              // residue tile output: [modulus][nx * 128][nt] bytes
};

// A grouped product: C blocks whose row blocks (C dims taken from A) and
// column blocks (C dims taken from B) form one dense grid, computed as one
// product over the union of their contracted blocks.  Row m of the group is
// tab[row_off + 5m .. +4] = (row block, its coordinates on the row dims, unused
// ones 0); columns likewise at col_off; tab[cell_off + R * ncb + S] is the
// DCrtCell of row block R and column block S, or -1 when that block is not
// computed by this contraction.
struct DCrtComp {
    int32_t rows, cols;           // C rows (side of A) and columns (side of B)
    int32_t ncb;                  // column blocks
    int32_t row_off, col_off, cell_off;
};
// Grouped products: a C block of a group, its offset and the C strides of
// its row dims (the C dims taken from A, in C order) and column dims; the row
// entries of DCrtComp give a row's block and its coordinates on those dims.
constexpr int kCrtSideDims = 4;
struct DCrtCell {
    int64_t c_off;
    int32_t ms[kCrtSideDims], ns[kCrtSideDims];
};

// Moduli of a modular contraction and its scaling (the constants of Garner's
// reconstruction are compile-time functions of the same moduli in crt.cu).
struct CrtParams {
    int32_t L;                    // number of moduli
    int32_t P;                    // bits of the scaled integer operands
    int32_t swap;                 // 1: MMA M side = the C columns (B operand)
    int32_t pad;
    int32_t m[kCrtMaxModuli];     // moduli, pairwise coprime, <= 256
    double minv_d[kCrtMaxModuli]; // 1 / m_i
};

// One operand cell of a grouped plain product: rows x K elements of a
// canonical block (row and k mappings of the pair's orbit transform, times
// coef) copied to buf[dst_off + r * ld + k].
struct DGather {
    int64_t src_off, dst_off;
    int32_t src;                  // 0: A arena, 1: B arena
    int32_t rows, K, ld, coef;
    int32_t nr, nk, pad;
    int32_t rext[kDevMaxSub], rstr[kDevMaxSub];
    int32_t kext[kDevMaxSub], kstr[kDevMaxSub];
};

// ---------------------------------------------------------------- element-wise

constexpr int kMaxTerms = 8;

// One destination block of a copy/add (or one A/B block pair of a dot
// product), seen as planes of A rows x B columns: the columns are the
// innermost destination dim, the rows dim q (the destination dim that is
// contiguous in a transposing source, else the next-to-innermost dim), and
// every other dim is an outer dim enumerating the planes.  Row r of the job
// is plane r / A, row r % A.
struct DJob {
    int64_t dst_off;
    int32_t nterms, term0;        // terms[term0 .. term0+nterms)
    int32_t A, B;                 // rows per plane (extent of dim q), columns
    int32_t dq;                   // destination stride of dim q
    int32_t nout;                 // outer dims, outermost first
    int32_t oext[kDevMaxOrder - 2], odst[kDevMaxOrder - 2];
    int32_t vec;                  // 16-byte accesses valid for every term
    int32_t seg, nseg;            // row mode: columns per item, column segments per row
    int32_t ra, nra;              // row mode: rows per item, row chunks per plane
    int32_t tiled;                // 1: 32x32 tiles staged through shared memory
    int32_t nta, ntb;             // tiled mode: tiles along the rows and the columns
};

struct DTerm {
    int64_t src_off;
    double coeff;
    int32_t src;                  // source tensor index
    int32_t sq, sb;               // source strides of dim q and of the columns
    int32_t tmode;                // tiled mode: 0 tile stored [row][col], 1 stored [col][row]
    int32_t osrc[kDevMaxOrder - 2];   // source strides of the outer dims
    int32_t toff, tld;            // tiled mode: tile offset (doubles) in shared memory, leading dim
    int32_t tvec, pad2;           // tiled mode, layout 0: 16-byte copies valid
};

// A range [row_begin, row_end) of one job's work items processed by one CTA:
// warp items ((plane * nra + chunk) * nseg + segment) in row mode, tiles
// ((plane * nta + ta) * ntb + tb) in tiled mode.
struct DUnit {
    int32_t job;
    int32_t pad;
    int64_t row_begin, row_end;
};

// ---------------------------------------------------------------- seeded inputs

// Counter-based test-input generator, identical on host and device.
// g(seed, x) is the centred sum of twelve 32-bit uniforms drawn from
// splitmix64 (Steele, Lea & Flood, OOPSLA 2014) keyed by the element's
// linear index in the full dense tensor: an integer in (-6*2^32, 6*2^32) with
// the variance of N(0,1) * 2^32 (the classic sum-of-12-uniforms normal
// approximation).  A symmetrised value is sum_{P in G} c_P * g(P x); the
// final double is that integer times scale * 2^-32, one correctly rounded
// multiply, so host and device produce the same bits.
__host__ __device__ inline uint64_t sm64_mix(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

__host__ __device__ inline int64_t seeded_int(uint64_t seed, uint64_t lin) {
    uint64_t key = sm64_mix(seed);
    uint64_t s = 0;
    for (int r = 0; r < 6; r++) {
        uint64_t h = sm64_mix(key + lin * 6u + (uint64_t)r);
        s += (h & 0xffffffffULL) + (h >> 32);
    }
    return (int64_t)s - (int64_t)(6ULL << 32);
}

// Symmetry group of the generator (full group closure, perm + coefficient).
struct DGenGroup {
    int32_t order;                 // tensor order
    int32_t ngroup;                // group elements
    int8_t perm[48][kDevMaxOrder]; // element permutations
    int8_t coeff[48];              // +1 / -1
    int64_t dims[kDevMaxOrder];    // full tensor extents
};

__host__ __device__ inline double seeded_value(const DGenGroup &g, uint64_t seed,
                                               double scale_2m32, const int64_t *x) {
    int64_t v = 0;
    for (int e = 0; e < g.ngroup; e++) {
        uint64_t lin = 0;
        for (int d = 0; d < g.order; d++) lin = lin * (uint64_t)g.dims[d] + (uint64_t)x[g.perm[e][d]];
        int64_t s = seeded_int(seed, lin);
        v += g.coeff[e] > 0 ? s : -s;
    }
#ifdef __CUDA_ARCH__
    return __dmul_rn((double)v, scale_2m32);
#else
    return (double)v * scale_2m32;
#endif
}

// ---------------------------------------------------------------- launchers

// Plain FP64 DMMA grouped contraction over all work items; partial tiles of
// k-split items go to ws (BM x BN doubles per slot).
// With dests (and drange, one index range of dests per C block), every C
// block's tile is added atomically to its destinations instead of being
// written (no k chunks: every item covers its whole k range).
cudaError_t launch_contract_fp64(const DTask *tasks, const DCBlock *cblks,
    const DItem *items, int32_t nitems, int32_t *counter, const double *a,
    const double *b, double *c, double *ws, int32_t add, int32_t tile_cfg, cudaStream_t s,
    const int2 *drange = nullptr, const DCBlock *dests = nullptr);
// Sums the partial tiles of every split tile in chunk order and writes (or
// adds) the scaled result into its C block.
cudaError_t launch_split_reduce(const DSplit *splits, int32_t nsplits, const DCBlock *cblks,
    const double *ws, int32_t bm, int32_t bn, double *c, int32_t add, cudaStream_t s);
int tile_cfg_bk(int cfg);

// Split-precision contraction: FP64 -> slice tile images, then the tcgen05
// grouped slice-product kernel with FP64 recombination.
cudaError_t launch_oz_split(int kind, const DPanel *panels, int32_t npanels, int32_t max_rows_pad,
    const double *a, const double *b, uint8_t *slices, int32_t *exps, int32_t S, cudaStream_t s);
// With dests (one range drange[cblk] per C block), each C block's tile is
// added atomically to its destinations (c zeroed before; add ignored); only
// for each kind's default slice count (INT8 and BF16 7, FP8 8).
cudaError_t launch_oz_gemm(int kind, const DPanel *panels, const uint8_t *slices, const DOzTask *tasks,
    const DCBlock *cblks, const DItem *items, int32_t nitems, const int32_t *exps, double *c,
    int32_t add, int32_t S, int32_t chunk_kb, int32_t *err, uint64_t wait_ns, cudaStream_t s,
    const int2 *drange = nullptr, const DCBlock *dests = nullptr);
// Per kind: first-slice bits, further-slice bits, element bytes, k elements
// per 64-byte k block, bound of one slice product.
void oz_kind_params(int kind, int *beta0, int *beta, int *esz, int *kbe, int64_t *maxprod);

// Modular split precision: exponent pass, residue pass, modular products,
// Garner recombination into FP64 C.
// Split passes work on units (panel, first row, rows, unused): at most 256
// rows of one panel.
// sample != 0: long rows of row-mapped units (crt_unit_sampled) contribute
// a sampled bound, one binade above the largest sampled magnitude.
cudaError_t launch_crt_exponents(const DCrtPanel *panels, const int4 *units, int32_t nunits,
    int32_t nx, int32_t ny, const double *a, const double *b, const int32_t *gidx, int32_t *ex,
    int32_t *ey, int32_t sample, cudaStream_t s);
bool crt_unit_sampled(const DCrtPanel &p, int unit_map);
int64_t crt_sampled_elems(const DCrtPanel &p);        // elements of one row the sampled pass reads
// Sets both exponent tables to "no element" (before the passes below).
cudaError_t launch_crt_fill(int32_t nx, int32_t ny, int32_t *ex, int32_t *ey, cudaStream_t s);

// Exponents and residues of the row families in one HBM read, in kernel
// shape 1-4 (units: crt_fuse_rows(shape) rows of one family, {family, first
// row, rows, 0}); ex/ey hold kNoExp before.
int crt_fuse_rows(int shape);
cudaError_t launch_crt_fused(int shape, const DCrtPanel *panels, const DCrtFamily *fams, const int32_t *famp,
    const int32_t *famt, const int4 *units, int32_t nunits, const double *a, const double *b,
    const int32_t *gidx, int32_t *ex, int32_t *ey, uint8_t *res, const CrtParams &cp, cudaStream_t s);
// sample != 0: sampled rows also form their exact exponents into ext / eyt
// (set to "no element" before); redo != 0: only the sampled rows whose exact
// exponent exceeds their bound run, with the exact exponent.
cudaError_t launch_crt_residues(const DCrtPanel *panels, const int4 *units, int32_t nunits,
    const double *a, const double *b, const int32_t *gidx, const int32_t *ex, const int32_t *ey,
    int32_t *ext, int32_t *eyt, int32_t sample, int32_t redo, uint8_t *res, const CrtParams &cp,
    cudaStream_t s);
// Products: ncta persistent CTAs, CTA b working through the items
// cta_items[j], j in [cta_items[b], cta_items[b + 1]).
cudaError_t launch_crt_gemm(const DCrtPanel *panels, const uint8_t *res, const DCrtTask *tasks,
    const DCrtItem *items, const int32_t *cta_items, int32_t ncta, uint8_t *out, const CrtParams &cp, int32_t *err,
    uint64_t wait_ns, int32_t stage_kb, cudaStream_t s);
// Destinations of a contraction's C blocks in another tensor (a two-term
// symmetrizer fused into the recombination): per C block of its own a range
// of dests (offset, index mapping; scale = the coefficient), at most
// kCrtMaxDests; per cell of a grouped product a range of gdcells with
// coefficients gdcoef.
constexpr int kCrtMaxDests = 8;
struct CrtDests {
    const int2 *drange;
    const DCBlock *dests;
    const int2 *gdrange;
    const DCrtCell *gdcells;
    const double *gdcoef;
};
// Garner recombination into C; each row's exponent is max(ex, ext) (the
// bound, or the exact exponent of a row the residue pass redid).  With dd,
// each element is added atomically to its destinations instead (c zeroed
// before; add ignored).
cudaError_t launch_crt_combine(const DCrtPanel *panels, const DCrtItem *items, int32_t nitems,
    const DCBlock *cblks, const DCrtComp *comps, const int32_t *ctab, const DCrtCell *cells,
    const uint8_t *out, const int32_t *gidx, const int32_t *ex, const int32_t *ey, const int32_t *ext, const int32_t *eyt, double *c,
    int32_t add, double scale, const CrtParams &cp, cudaStream_t s, const CrtDests *dd = nullptr);

// Grouped plain products: operand cells into dense group panels (units:
// piece, first row, rows), and the dense group results into the C blocks
// (units: group, result row).
cudaError_t launch_gather_cells(const DGather *pieces, const int4 *units, int32_t nunits,
    const double *a, const double *b, double *buf, cudaStream_t s);
cudaError_t launch_scatter_groups(const DCrtComp *comps, const int64_t *res_off, const int32_t *ctab,
    const DCrtCell *cells, const int2 *units, int32_t nunits, const double *buf, double *c,
    double scale, int32_t add, cudaStream_t s);
// The group results added atomically (into a zeroed r) to the destinations
// of each cell: dcells[drange[cell].x .. .y) times dcoef.
cudaError_t launch_scatter_groups_dest(const DCrtComp *comps, const int64_t *res_off, const int32_t *ctab,
    const int2 *drange, const DCrtCell *dcells, const double *dcoef, const int2 *units, int32_t nunits,
    const double *buf, double *r, double scale, cudaStream_t s);

// Element-wise transfer kernels.  max_terms bounds nterms and tile_bytes the
// shared-memory tiles of any tiled-mode job.
// Units are ordered row-mode units first (nrow of them), then tiled-mode
// units (ntiled); the dot product leaves one partial sum per unit.
cudaError_t launch_transfer(const DJob *jobs, const DTerm *terms, const DUnit *units,
    int32_t nrow, int32_t ntiled, int32_t max_terms, int32_t tile_bytes, const double *const *srcs,
    double *dst, int32_t accumulate, double beta, cudaStream_t s);
cudaError_t launch_dot(const DJob *jobs, const DTerm *terms, const DUnit *units,
    int32_t nrow, int32_t ntiled, int32_t tile_bytes, const double *a, const double *b,
    double *partials, double *out, cudaStream_t s);
cudaError_t launch_scale(double *x, int64_t n, double c, cudaStream_t s);
cudaError_t launch_fill_seeded(double *arena, const int64_t *blk_off,
    const int64_t *blk_start, const int32_t *blk_ext, int32_t nblk, int32_t order,
    const DGenGroup &g, uint64_t seed, double scale_2m32, cudaStream_t s);
cudaError_t launch_denominator(double *arena, const int64_t *blk_off,
    const int64_t *blk_start, const int32_t *blk_ext, int32_t nblk,
    const double *eps, const int64_t *eps_off, int32_t nocc, cudaStream_t s);

}  // namespace ltg
