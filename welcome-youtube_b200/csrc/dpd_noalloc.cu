// dpd_noalloc.cu -- the cell sort for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: code that runs inside
// another framework's operator or plugin hook (an XLA or TensorFlow custom
// call, a TensorRT plugin's enqueue, a PyTorch op under a memory-pool guard)
// owns no allocator of its own there, and cudaMalloc / cudaFree synchronise the
// whole device, which such hooks must not do.  The handle API (dpd_create) does
// allocate, so it is closed to them.  dpd_sort_cells_noalloc gives them the
// stable cell sort of bead positions with every scratch buffer in one
// file-scope device array of fixed size (below): the caller passes device
// inputs and outputs only, and nothing is allocated or freed, ever.
//
// Limits: at most DPD_NOALLOC_MAX_BEADS beads and DPD_NOALLOC_MAX_CELLS cells
// per call (larger requests are refused with DPD_E_ARG).  The array takes
// (2 * MAX_CELLS + MAX_BEADS + 2048) * 4 bytes = 8.0 MiB on every GPU that loads
// the library, for as long as the process lives.  All calls share the array:
// two calls whose work overlaps on the GPU (different streams, or different
// host threads on one device) race and corrupt each other; calls on one stream
// in order are safe.  The first call on each device looks up the array's
// device address (cudaGetSymbolAddress), so make that first call before any
// stream capture begins.
#include <cmath>
#include <cstring>
#include <cuda_runtime.h>

#include "../../include/dpd.h"

#define NA_TPB 256
#define NA_SCAN_BLOCK 2048  // cells per scan block (8 per thread)
#define NA_MAX_DEVICES 64

// scratch layout (32-bit words): key[MAX_BEADS] | count[MAX_CELLS] | fill[MAX_CELLS] | bsum[2048]
#define NA_WORDS (2u * DPD_NOALLOC_MAX_CELLS + DPD_NOALLOC_MAX_BEADS + 2048u)
static __device__ __align__(256) unsigned int g_noalloc_scratch[NA_WORDS];

// device address of g_noalloc_scratch on each device, looked up once per device
static unsigned int *g_scratch_ptr[NA_MAX_DEVICES];

static int noalloc_setup(int dev, unsigned int **out) {
    if (dev < 0 || dev >= NA_MAX_DEVICES) return DPD_E_ARG;
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return DPD_E_CUDA;
        g_scratch_ptr[dev] = (unsigned int *)p;
    }
    *out = g_scratch_ptr[dev];
    return DPD_OK;
}

// cell of a position as in the handle API: ncx = ncy = floor(L), column-major,
// the product taken in FP64 (the reference's cell_of_pos with nsub = 1)
__device__ __forceinline__ unsigned na_cell(float x, float y, int nc, double ics) {
    int cx = (int)((double)x * ics), cy = (int)((double)y * ics);
    cx = cx >= nc ? nc - 1 : (cx < 0 ? 0 : cx);
    cy = cy >= nc ? nc - 1 : (cy < 0 ? 0 : cy);
    return (unsigned)(cx * nc + cy);
}

__global__ void k_na_count(const float *x, const float *y, int n, int nc, double ics, unsigned *key,
                           unsigned *count) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned c = na_cell(x[i], y[i], nc, ics);
        key[i] = c;
        atomicAdd(count + c, 1u);
    }
}

// exclusive scan, pass 1: block-local scan of NA_SCAN_BLOCK cells into cstart, block totals into bsum
__global__ void k_na_scan1(const unsigned *count, int32_t *cstart, unsigned *bsum, int C) {
    __shared__ unsigned ws[NA_TPB / 32];
    const int base = blockIdx.x * NA_SCAN_BLOCK + threadIdx.x * 8;
    unsigned v[8], s = 0;
    for (int k = 0; k < 8; k++) {
        v[k] = base + k < C ? count[base + k] : 0u;
        s += v[k];
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned x = s;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += t;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    unsigned before = 0;
    for (int k = 0; k < w; k++) before += ws[k];
    unsigned ex = before + x - s;
    for (int k = 0; k < 8; k++) {
        if (base + k < C) cstart[base + k] = (int32_t)ex;
        ex += v[k];
    }
    if (threadIdx.x == NA_TPB - 1) bsum[blockIdx.x] = before + x;
}

// pass 2: add the totals of earlier blocks; copy to the placement cursor; cstart[C] = n
__global__ void k_na_scan2(int32_t *cstart, unsigned *fill, const unsigned *bsum, int C, int nblocks) {
    __shared__ unsigned pre;
    if (threadIdx.x == 0) {
        unsigned p = 0;
        for (int k = 0; k < (int)blockIdx.x; k++) p += bsum[k];
        pre = p;
        if ((int)blockIdx.x == nblocks - 1) cstart[C] = (int32_t)(p + bsum[blockIdx.x]);
    }
    __syncthreads();
    const int base = blockIdx.x * NA_SCAN_BLOCK + threadIdx.x * 8;
    for (int k = 0; k < 8; k++)
        if (base + k < C) {
            const int32_t v = cstart[base + k] + (int32_t)pre;
            cstart[base + k] = v;
            fill[base + k] = (unsigned)v;
        }
}

__global__ void k_na_place(const unsigned *key, unsigned *fill, int32_t *order, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        order[atomicAdd(fill + key[i], 1u)] = i;
}

// stable order inside each cell: ascending input index (insertion sort; cells hold a few beads)
__global__ void k_na_cellfix(const int32_t *cstart, int32_t *order, int C) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x) {
        const int s = cstart[c], e = cstart[c + 1];
        for (int k = s + 1; k < e; k++) {
            const int32_t t = order[k];
            int q = k - 1;
            while (q >= s && order[q] > t) {
                order[q + 1] = order[q];
                q--;
            }
            order[q + 1] = t;
        }
    }
}

extern "C" int dpd_sort_cells_noalloc(const float *x, const float *y, int32_t n, double L, int32_t *cstart,
                                      int32_t *order, void *stream) {
    if (!x || !y || !cstart || !order || n < 1 || !(L >= 3.0) || !std::isfinite(L)) return DPD_E_ARG;
    const float Lf = (float)L;
    const int nc = (int)std::floor((double)Lf);
    const long long C = (long long)nc * nc;
    if (n > DPD_NOALLOC_MAX_BEADS || C > DPD_NOALLOC_MAX_CELLS) return DPD_E_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return DPD_E_CUDA;
    unsigned *scratch = nullptr;
    const int rc = noalloc_setup(dev, &scratch);
    if (rc != DPD_OK) return rc;
    unsigned *key = scratch, *count = key + DPD_NOALLOC_MAX_BEADS, *fill = count + DPD_NOALLOC_MAX_CELLS,
             *bsum = fill + DPD_NOALLOC_MAX_CELLS;
    cudaStream_t s = (cudaStream_t)stream;
    const double ics = nc / (double)Lf;
    const int nb = (int)((C + NA_SCAN_BLOCK - 1) / NA_SCAN_BLOCK);
    const int gb = (n + NA_TPB - 1) / NA_TPB, gc = (int)((C + NA_TPB - 1) / NA_TPB);
    // counts must start at zero: the array keeps the previous call's contents
    if (cudaMemsetAsync(count, 0, (size_t)C * sizeof(unsigned), s) != cudaSuccess) return DPD_E_CUDA;
    k_na_count<<<gb, NA_TPB, 0, s>>>(x, y, n, nc, ics, key, count);
    k_na_scan1<<<nb, NA_TPB, 0, s>>>(count, cstart, bsum, (int)C);
    k_na_scan2<<<nb, NA_TPB, 0, s>>>(cstart, fill, bsum, (int)C, nb);
    k_na_place<<<gb, NA_TPB, 0, s>>>(key, fill, order, n);
    k_na_cellfix<<<gc, NA_TPB, 0, s>>>(cstart, order, (int)C);
    return cudaGetLastError() == cudaSuccess ? DPD_OK : DPD_E_CUDA;
}
