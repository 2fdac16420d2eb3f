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
// stream capture begins.  The looked-up address is kept for the life of the
// process: after a cudaDeviceReset of a device, this entry point must not be
// called on that device again.
//
// The work is bounded whatever the positions.  Cells of up to 16 beads are
// ordered by one thread each; a crowded cell (more than 16) is listed and
// ordered by a whole CTA: up to NA_SORT_MAX beads by a bitonic sort in shared
// memory, more by a compaction of the input indices whose cell it is (one pass
// over the n keys; at most n / NA_SORT_MAX cells take this path).  So even n
// beads in a single cell, e.g. zero-initialised positions, cost one pass.
#include <atomic>
#include <climits>
#include <cmath>
#include <cstring>
#include <cuda_runtime.h>

#include "../../include/dpd.h"

#define NA_TPB 256
#define NA_SCAN_BLOCK 2048  // cells per scan block (8 per thread)
#define NA_MAX_DEVICES 64
#define NA_SMALL 16         // cells up to this size are ordered by one thread
#define NA_SORT_MAX 4096    // crowded cells up to this size: bitonic sort in shared memory
#define NA_CROWD_GRID 512   // CTAs of k_na_crowded (each takes listed cells in turn)

// scratch layout (32-bit words): key[MAX_BEADS] | count[MAX_CELLS] | fill[MAX_CELLS] | misc[2048]
//   misc[0, 256): scan block totals; misc[NA_CROWD_CTR]: crowded cells listed.
//   count[] is free once scanned and then holds the list of crowded cells.
#define NA_WORDS (2u * DPD_NOALLOC_MAX_CELLS + DPD_NOALLOC_MAX_BEADS + 2048u)
#define NA_CROWD_CTR 2047
static __device__ __align__(256) unsigned int g_noalloc_scratch[NA_WORDS];

// device address of g_noalloc_scratch on each device, looked up once per device
static std::atomic<unsigned int *> g_scratch_ptr[NA_MAX_DEVICES];

static int noalloc_setup(int dev, unsigned int **out) {
    if (dev < 0 || dev >= NA_MAX_DEVICES) return DPD_E_ARG;
    unsigned int *p = g_scratch_ptr[dev].load(std::memory_order_acquire);
    if (!p) {
        void *q = nullptr;
        if (cudaGetSymbolAddress(&q, g_noalloc_scratch) != cudaSuccess || !q) return DPD_E_CUDA;
        p = (unsigned int *)q;
        g_scratch_ptr[dev].store(p, std::memory_order_release);  // racing threads store the same address
    }
    *out = p;
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
__global__ void k_na_scan2(int32_t *cstart, unsigned *fill, unsigned *bsum, int C, int nblocks) {
    __shared__ unsigned pre;
    if (blockIdx.x == 0 && threadIdx.x == 0) bsum[NA_CROWD_CTR] = 0u;  // the crowded list of this call starts empty
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

// stable order inside each cell: ascending input index.  Up to NA_SMALL beads
// here (insertion sort, at most 120 moves); larger cells go to the crowded list.
__global__ void k_na_cellfix(const int32_t *cstart, int32_t *order, int C, unsigned *crowd, unsigned *ncrowd) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x) {
        const int s = cstart[c], e = cstart[c + 1];
        if (e - s > NA_SMALL) {
            crowd[atomicAdd(ncrowd, 1u)] = (unsigned)c;
            continue;
        }
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

// block-wide exclusive scan of one value per thread (NA_TPB threads)
__device__ __forceinline__ unsigned na_block_scan(unsigned v, unsigned *total) {
    __shared__ unsigned ws[NA_TPB / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += t;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    unsigned before = 0, all = 0;
    for (int k = 0; k < NA_TPB / 32; k++) {
        before += k < w ? ws[k] : 0u;
        all += ws[k];
    }
    __syncthreads();  // ws is reused by the next call
    *total = all;
    return before + x - v;
}

// one CTA per listed crowded cell, in turn.  Up to NA_SORT_MAX beads: bitonic
// sort of the cell's input indices in shared memory.  More: the cell's slots
// are rewritten as the compaction of {i : key[i] == c} in ascending i, one pass
// over the n keys (so at most n / NA_SORT_MAX such passes in all).
__global__ void __launch_bounds__(NA_TPB) k_na_crowded(const int32_t *cstart, int32_t *order, const unsigned *key,
                                                       int n, const unsigned *crowd, const unsigned *ncrowd) {
    __shared__ int32_t v[NA_SORT_MAX];
    const int nl = (int)*ncrowd;
    for (int k = blockIdx.x; k < nl; k += gridDim.x) {
        const unsigned c = crowd[k];
        const int s = cstart[c], m = cstart[c + 1] - s;
        if (m <= NA_SORT_MAX) {
            int P = 1;
            while (P < m) P <<= 1;
            for (int i = threadIdx.x; i < P; i += NA_TPB) v[i] = i < m ? order[s + i] : INT_MAX;
            __syncthreads();
            for (int kk = 2; kk <= P; kk <<= 1)
                for (int j = kk >> 1; j > 0; j >>= 1) {
                    for (int i = threadIdx.x; i < P; i += NA_TPB) {
                        const int l = i ^ j;
                        if (l > i) {
                            const int32_t a = v[i], b = v[l];
                            if (((i & kk) == 0) ? (a > b) : (a < b)) {
                                v[i] = b;
                                v[l] = a;
                            }
                        }
                    }
                    __syncthreads();
                }
            for (int i = threadIdx.x; i < m; i += NA_TPB) order[s + i] = v[i];
        } else {
            unsigned run = 0;
            for (int base = 0; base < n; base += NA_TPB * 16) {  // 16 consecutive keys per thread
                const int i0 = base + threadIdx.x * 16;
                unsigned f = 0;
                if (i0 + 16 <= n) {
                    const uint4 *kp = reinterpret_cast<const uint4 *>(key + i0);  // key is 256-byte aligned
                    for (int q = 0; q < 4; q++) {
                        const uint4 w = kp[q];
                        f |= (unsigned)(w.x == c) << (4 * q) | (unsigned)(w.y == c) << (4 * q + 1) |
                             (unsigned)(w.z == c) << (4 * q + 2) | (unsigned)(w.w == c) << (4 * q + 3);
                    }
                } else {
                    for (int q = 0; q < 16; q++) f |= (i0 + q < n && key[i0 + q] == c) ? (1u << q) : 0u;
                }
                unsigned total;
                unsigned ex = na_block_scan((unsigned)__popc(f), &total);
                for (int q = 0; q < 16; q++)
                    if (f & (1u << q)) order[s + (int)(run + ex++)] = i0 + q;
                run += total;
            }
        }
        __syncthreads();  // v[] and the scan words are reused by the next listed cell
    }
}

extern "C" int dpd_sort_cells_noalloc(const float *x, const float *y, int32_t n, double L, int32_t *cstart,
                                      int32_t *order, void *stream) {
    if (!x || !y || !cstart || !order || n < 1 || !(L >= 3.0) || !std::isfinite(L)) return DPD_E_ARG;
    const float Lf = (float)L;
    const int nc = (int)std::floor((double)Lf);
    // the grid is floor of the FP32 box side, as in the handle API; an L whose
    // rounding to FP32 moves floor(L) (31.9999999 -> 32.0f) is refused, so that
    // cstart always holds floor(L)^2 + 1 entries
    if ((double)nc != std::floor(L)) return DPD_E_ARG;
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
    k_na_cellfix<<<gc, NA_TPB, 0, s>>>(cstart, order, (int)C, count, bsum + NA_CROWD_CTR);
    k_na_crowded<<<NA_CROWD_GRID, NA_TPB, 0, s>>>(cstart, order, key, n, count, bsum + NA_CROWD_CTR);
    return cudaGetLastError() == cudaSuccess ? DPD_OK : DPD_E_CUDA;
}
