// dpd_cells.cu -- cell detection in one snapshot on the GPU: the reference's
// detect() (cel/tools/cells.py:331-611) with every per-bead and per-pixel stage
// on the device and the same results.
//
// Stages, each a few grid-wide passes:
//  1. molecules: union-find over the bonds between lipid beads (H, T); a
//     molecule is numbered by the rank of its lowest bead, as
//     connected_components numbers components (cells.py:68-86);
//  2. tail contacts: T beads binned in cells of side >= r_tail, pairs with
//     distance <= r_tail (periodic, as the reference's KD-tree measures it);
//     aggregates: union-find over the molecules, numbered by their lowest
//     molecule (cells.py:345-366);
//  3. unwrapping of every aggregate of at least min_membrane_lipids molecules:
//     a level-synchronous breadth-first walk from its lowest bead that visits
//     the beads in the order scipy's breadth_first_order visits them (per
//     level, a bead is reached from the earliest bead of the previous level,
//     out-neighbours before in-neighbours, each list in index order), so the
//     FP64 sums of minimum-image steps equal the reference's bit for bit;
//     the wrap test on every edge (cells.py:89-133);
//  4. holes: the aggregate's beads stamped as disks on a pixel grid, solvent
//     labelled with 4-connectivity by a union-find over pixels.  Aggregates
//     that do not wrap use their own bounding box (holes: components that do
//     not touch the border, cells.py:192-201); wrapping ones the periodic
//     grid, where each pixel carries its image offset relative to its root,
//     so a component that meets itself with a non-zero offset wraps the torus
//     and every other one is an enclosed hole, unwrapped to the copy whose
//     centroid lies in the box (cells.py:204-297);
//  5. lumens painted largest first on the global label grid, their contents
//     counted, the bulk medium found (the largest periodic solvent component
//     of all lipids' stamps, and any of >= 25 %), the distance from each
//     lumen's boundary pixels to it (exact within the window the reference
//     searches), the aqueous and exposure tests (cells.py:406-459);
//  6. wall lipids: each lipid of an aggregate with lumens is assigned to the
//     lumen whose nearest boundary pixel centre is closest, per molecule by
//     its closest bead; leaflet counts of the heads (cells.py:470-537);
//  7. per cell: centroid, covariance and convex hull of the lumen pixels
//     (hull from each pixel row's two ends), the bilayer test and the final
//     numbering (cells.py:539-611).
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "dpd_internal.h"

struct dpd_cells {
    double h = 0;
    int64_t ng = 0, n = 0;
    int64_t summary[6] = {0, 0, 0, 0, 0, 0};
    std::vector<int64_t> aggs;  // 4 per membrane
    std::vector<double> cells;  // DPD_CELL_COLS per cell
    // on the device until fetched: label grid (ng x ng), per-bead cell, molecule, aggregate
    int32_t *label = nullptr, *bead_cell = nullptr, *mol = nullptr, *bead_agg = nullptr;
    ~dpd_cells() {
        for (int32_t *p : {label, bead_cell, mol, bead_agg})
            if (p) cudaFree(p);
    }
};

namespace dpd_cells_impl {

constexpr int TPB = 256;
constexpr int TW = 0, TH = 1, TT = 2, TN = 3, TKA = 4, TKB = 5, TZ = 6;
constexpr int MAXIT = 1 << 30;    // bound of a union-find walk (parents only decrease)
constexpr int MAXRETRY = 1 << 14; // bound of a union's compare-and-swap retries
constexpr int KEY_BIAS = 1 << 19; // unwrapped pixel coordinates in 20-bit key fields

struct Fail {
    int code;
    std::string msg;
};

#define CU(call)                                                                                 \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) throw Fail{DPD_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

template <class F>
__global__ void __launch_bounds__(TPB) k_each(long long n, F f) {
    const long long i = (long long)blockIdx.x * TPB + threadIdx.x;
    if (i < n) f(i);
}

struct Ctx {
    cudaStream_t s = nullptr;
    std::vector<void *> mem;
    int *err = nullptr;  // device flags: 1 union retries exhausted, 2 inconsistent torus roots, 4 key range
    void *tmp = nullptr;  // CUB scratch, grown on demand and kept for the whole call
    size_t tmp_bytes = 0;
    long long *pin = nullptr;  // pinned host words for small read-backs
    void init() {
        CU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        CU(cudaMallocHost((void **)&pin, 4 * sizeof(long long)));
        // stream-ordered allocations from the device's default pool, which keeps
        // freed memory for the next call instead of returning it (a free then
        // needs no device synchronisation)
        int dev = 0;
        cudaMemPool_t pool;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            unsigned long long keep = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        cudaGetLastError();
        err = zeros<int>(1);
    }
    ~Ctx() {
        for (void *p : mem) cudaFreeAsync(p, s);
        if (s) cudaStreamSynchronize(s);
        if (pin) cudaFreeHost(pin);
        if (s) cudaStreamDestroy(s);
    }
    void *scratch(size_t bytes) {
        if (bytes > tmp_bytes) {
            if (tmp) release(tmp);
            tmp = alloc<char>(bytes + bytes / 2);
            tmp_bytes = bytes + bytes / 2;
        }
        return tmp;
    }
    template <class T> T *alloc(size_t n) {
        void *p = nullptr;
        if (cudaMallocAsync(&p, std::max<size_t>(n, 1) * sizeof(T), s) != cudaSuccess) {
            cudaGetLastError();
            throw Fail{DPD_E_NOMEM, "cell detection: device allocation of " + std::to_string(n * sizeof(T)) +
                                        " bytes failed"};
        }
        mem.push_back(p);
        return (T *)p;
    }
    void adopt(void *p) {  // the caller keeps p: it is not freed with the context
        auto it = std::find(mem.begin(), mem.end(), p);
        if (it != mem.end()) mem.erase(it);
    }
    void release(void *p) {
        auto it = std::find(mem.begin(), mem.end(), p);
        if (it == mem.end()) return;
        CU(cudaFreeAsync(p, s));
        mem.erase(it);
    }
    template <class T> T *fill(size_t n, int byte) {
        T *p = alloc<T>(n);
        CU(cudaMemsetAsync(p, byte, std::max<size_t>(n, 1) * sizeof(T), s));
        return p;
    }
    template <class T> T *zeros(size_t n) { return fill<T>(n, 0); }
    template <class T> T *upload(const T *h, size_t n) {
        T *p = alloc<T>(n);
        if (n) CU(cudaMemcpyAsync(p, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
        CU(cudaStreamSynchronize(s));
        return p;
    }
    template <class T> T *upload(const std::vector<T> &v) { return upload(v.data(), v.size()); }
    template <class T> std::vector<T> download(const T *d, size_t n) {
        std::vector<T> v(n);
        if (n) CU(cudaMemcpyAsync(v.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        return v;
    }
    template <class T> T get(const T *d) {
        T v;
        CU(cudaMemcpyAsync(&v, d, sizeof(T), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        return v;
    }
    template <class F> void each(long long n, F f) {
        if (n <= 0) return;
        k_each<<<(unsigned)((n + TPB - 1) / TPB), TPB, 0, s>>>(n, f);
        CU(cudaGetLastError());
    }
    void check_flags(const char *where) {
        const int e = get(err);
        if (e) throw Fail{DPD_E_STATE, std::string("cell detection: ") + where + ": " +
                                           (e & 1 ? "union-find retries exhausted"
                                                  : e & 2 ? "inconsistent periodic labels" : "a hole exceeds the key range")};
    }
};

// exclusive prefix sum of n values; returns the total
template <class T> T scan(Ctx &c, const T *in, T *out, long long n) {
    if (n <= 0) return 0;
    size_t tb = 0;
    CU(cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, n, c.s));
    void *t = c.scratch(tb);
    CU(cub::DeviceScan::ExclusiveSum(t, tb, in, out, n, c.s));
    T *h = (T *)c.pin;
    CU(cudaMemcpyAsync(h, out + n - 1, sizeof(T), cudaMemcpyDeviceToHost, c.s));
    CU(cudaMemcpyAsync(h + 1, in + n - 1, sizeof(T), cudaMemcpyDeviceToHost, c.s));
    CU(cudaStreamSynchronize(c.s));
    return h[0] + h[1];
}

struct MaxOp {
    __device__ __forceinline__ int operator()(int a, int b) const { return a > b ? a : b; }
};

// inclusive running maximum: with key[p] = p at the start of each run of a row
// and -1 elsewhere, every pixel gets the first pixel of its run
void max_scan(Ctx &c, const int *in, int *out, long long n) {
    if (n <= 0) return;
    size_t tb = 0;
    CU(cub::DeviceScan::InclusiveScan(nullptr, tb, in, out, MaxOp(), n, c.s));
    void *t = c.scratch(tb);
    CU(cub::DeviceScan::InclusiveScan(t, tb, in, out, MaxOp(), n, c.s));
}

// the indices i < n with flag[i] == 1, increasing
int select_flags(Ctx &c, const int *flag, int n, int **out) {
    int *pos = c.alloc<int>(n);
    const int cnt = scan(c, flag, pos, (long long)n);
    int *idx = c.alloc<int>(cnt);
    c.each(n, [=] __device__(long long i) {
        if (flag[i]) idx[pos[i]] = (int)i;
    });
    c.release(pos);
    *out = idx;
    return cnt;
}

// stable sort of (key, value) pairs by key
void sort_pairs(Ctx &c, int *key, int *val, int n, int end_bit) {
    if (n <= 1) return;
    int *k2 = c.alloc<int>(n), *v2 = c.alloc<int>(n);
    size_t tb = 0;
    CU(cub::DeviceRadixSort::SortPairs(nullptr, tb, key, k2, val, v2, n, 0, end_bit, c.s));
    void *t = c.scratch(tb);
    CU(cub::DeviceRadixSort::SortPairs(t, tb, key, k2, val, v2, n, 0, end_bit, c.s));
    CU(cudaMemcpyAsync(key, k2, n * sizeof(int), cudaMemcpyDeviceToDevice, c.s));
    CU(cudaMemcpyAsync(val, v2, n * sizeof(int), cudaMemcpyDeviceToDevice, c.s));
    c.release(k2);
    c.release(v2);
}

void sort_keys(Ctx &c, unsigned long long *key, int n, int end_bit) {
    if (n <= 1) return;
    unsigned long long *k2 = c.alloc<unsigned long long>(n);
    size_t tb = 0;
    CU(cub::DeviceRadixSort::SortKeys(nullptr, tb, key, k2, n, 0, end_bit, c.s));
    void *t = c.scratch(tb);
    CU(cub::DeviceRadixSort::SortKeys(t, tb, key, k2, n, 0, end_bit, c.s));
    CU(cudaMemcpyAsync(key, k2, (size_t)n * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, c.s));
    c.release(k2);
}

int bits_for(long long v) {
    int b = 1;
    while ((1ll << b) <= v) b++;
    return b;
}

// ---------------------------------------------------------------- device helpers

__device__ __forceinline__ long long pmod(long long a, long long m) {
    const long long r = a % m;
    return r < 0 ? r + m : r;
}

// numpy's d - L * np.round(d / L) (cells.py:64-65)
__device__ __forceinline__ double minimg(double d, double L) {
    return __dsub_rn(d, __dmul_rn(L, rint(__ddiv_rn(d, L))));
}

// the KD-tree's periodic coordinate difference (scipy cKDTree with boxsize)
__device__ __forceinline__ double kd_wrap(double d, double L) {
    const double hb = 0.5 * L;
    return d < -hb ? __dadd_rn(d, L) : (d > hb ? __dsub_rn(d, L) : d);
}

__device__ __forceinline__ double sq2(double dx, double dy) { return __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)); }

__device__ __forceinline__ unsigned long long dkey(double v) {  // order-preserving key of a double
    const unsigned long long u = (unsigned long long)__double_as_longlong(v);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
inline double dkey_inv(unsigned long long k) {
    const unsigned long long u = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    double v;
    std::memcpy(&v, &u, sizeof v);
    return v;
}

__device__ __forceinline__ int uf_find(int *par, int i) {
    for (int it = 0; it < MAXIT; it++) {
        const int p = __ldcg(par + i);
        if (p == i) return i;
        const int g = __ldcg(par + p);
        if (g != p) atomicCAS(par + i, p, g);
        i = g;
    }
    return i;
}

// links the larger root under the smaller: every set ends with its lowest index as root
__device__ __forceinline__ void uf_union(int *par, int a, int b, int *err) {
    for (int it = 0; it < MAXRETRY; it++) {
        a = uf_find(par, a);
        b = uf_find(par, b);
        if (a == b) return;
        const int lo = a < b ? a : b, hi = a < b ? b : a;
        if (atomicCAS(par + hi, hi, lo) == hi) return;
        a = lo;
        b = hi;
    }
    atomicOr(err, 1);
}

// after the unions: a run start points straight at its root (only this
// thread writes entry i; the others' entries it reads only ever shorten), so a
// pixel then reaches its root in two hops whatever the order of the links was
__device__ __forceinline__ void uf_flatten(int *par, int i) {
    int x = __ldcg(par + i);
    for (int it = 0; it < MAXIT; it++) {
        const int y = __ldcg(par + x);
        if (y == x) break;
        x = y;
        par[i] = x;
    }
}

// weighted union-find on the periodic grid: a word holds the parent (low 32
// bits) and the node's image offset relative to it (two int16); a root's word
// is (itself, 0, 0)
__device__ __forceinline__ unsigned long long wpack(int p, int ox, int oy) {
    return (unsigned long long)(unsigned)p | ((unsigned long long)(unsigned short)(short)ox << 32) |
           ((unsigned long long)(unsigned short)(short)oy << 48);
}
__device__ __forceinline__ int wpar(unsigned long long w) { return (int)(unsigned)w; }
__device__ __forceinline__ int wox(unsigned long long w) { return (short)(unsigned short)(w >> 32); }
__device__ __forceinline__ int woy(unsigned long long w) { return (short)(unsigned short)(w >> 48); }

// the weighted form of uf_flatten: entry i gets its root and its offset to it
__device__ __forceinline__ void wflatten(unsigned long long *par, int i) {
    unsigned long long w = __ldcg(par + i);
    int x = (int)(unsigned)w, ox = (short)(unsigned short)(w >> 32), oy = (short)(unsigned short)(w >> 48);
    for (int it = 0; it < MAXIT; it++) {
        const unsigned long long v = __ldcg(par + x);
        const int y = (int)(unsigned)v;
        if (y == x) break;
        ox += (short)(unsigned short)(v >> 32);
        oy += (short)(unsigned short)(v >> 48);
        x = y;
        par[i] = (unsigned long long)(unsigned)x | ((unsigned long long)(unsigned short)(short)ox << 32) |
                 ((unsigned long long)(unsigned short)(short)oy << 48);
    }
}

__device__ __forceinline__ int wfind(unsigned long long *par, int i, int &ox, int &oy) {
    ox = 0;
    oy = 0;
    for (int it = 0; it < MAXIT; it++) {
        const unsigned long long w = __ldcg(par + i);
        const int p = wpar(w);
        if (p == i) return i;
        const unsigned long long wp = __ldcg(par + p);
        const int g = wpar(wp);
        if (g == p) {
            ox += wox(w);
            oy += woy(w);
            return p;
        }
        const int nx = wox(w) + wox(wp), ny = woy(w) + woy(wp);
        atomicCAS(par + i, w, wpack(g, nx, ny));  // halving: i skips to its grandparent
        ox += nx;
        oy += ny;
        i = g;
    }
    return i;
}

// joins a and b where b's image is a's plus (sx, sy)
__device__ __forceinline__ void wunion(unsigned long long *par, int a, int b, int sx, int sy, int *err) {
    for (int it = 0; it < MAXRETRY; it++) {
        int ax, ay, bx, by;
        const int ra = wfind(par, a, ax, ay), rb = wfind(par, b, bx, by);
        if (ra == rb) return;
        const int dx = sx + ax - bx, dy = sy + ay - by;  // offset of rb relative to ra
        if (ra < rb) {
            if (atomicCAS(par + rb, wpack(rb, 0, 0), wpack(ra, dx, dy)) == wpack(rb, 0, 0)) return;
        } else {
            if (atomicCAS(par + ra, wpack(ra, 0, 0), wpack(rb, -dx, -dy)) == wpack(ra, 0, 0)) return;
        }
    }
    atomicOr(err, 1);
}

// counter[key] += 1 with one atomic per distinct key among the warp's active
// threads: most pixels of a labelling pass add to the same few roots
template <class T> __device__ __forceinline__ void agg_inc(T *counter, int key) {
    const unsigned grp = __match_any_sync(__activemask(), key);
    if ((int)(threadIdx.x & 31) == __ffs(grp) - 1) atomicAdd(counter + key, (T)__popc(grp));
}

__device__ __forceinline__ int find_seg(const long long *base, int nseg, long long p) {  // base[s] <= p < base[s+1]
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (base[mid] <= p)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ bool is_solvent_type(int t) {
    return t == TW || t == TN || t == TKA || t == TKB || t == TZ;
}

// ---------------------------------------------------------------- host pieces

struct Lumen {
    int agg;
    const int2 *src;  // pixel list on the device (unwrapped global coordinates, raster order)
    long long cnt;
    double area_raw;
    bool wraps;
};

// Python's float % for a positive modulus
double py_mod(double v, double m) {
    double r = std::fmod(v, m);
    if (r != 0.0) {
        if ((r < 0) != (m < 0)) r += m;
    } else {
        r = std::copysign(0.0, m);
    }
    return r;
}

// twice the area of the convex hull of integer points (Andrew's monotone chain)
long long hull_area2(std::vector<std::pair<long long, long long>> &pts) {
    std::sort(pts.begin(), pts.end());
    pts.erase(std::unique(pts.begin(), pts.end()), pts.end());
    const size_t n = pts.size();
    if (n < 3) return 0;
    auto cross = [](const std::pair<long long, long long> &o, const std::pair<long long, long long> &a,
                    const std::pair<long long, long long> &b) {
        return (a.first - o.first) * (b.second - o.second) - (a.second - o.second) * (b.first - o.first);
    };
    std::vector<std::pair<long long, long long>> hull(2 * n);
    size_t k = 0;
    for (size_t i = 0; i < n; i++) {
        while (k >= 2 && cross(hull[k - 2], hull[k - 1], pts[i]) <= 0) k--;
        hull[k++] = pts[i];
    }
    for (size_t i = n - 1, t = k + 1; i > 0; i--) {
        while (k >= t && cross(hull[k - 2], hull[k - 1], pts[i - 1]) <= 0) k--;
        hull[k++] = pts[i - 1];
    }
    hull.resize(k - 1);
    long long a2 = 0;
    for (size_t i = 0; i < hull.size(); i++) {
        const auto &p = hull[i], &q = hull[(i + 1) % hull.size()];
        a2 += p.first * q.second - q.first * p.second;
    }
    return a2 < 0 ? -a2 : a2;
}

void detect(const dpd_cells_cfg &cfg, double L, long long n64, const double *hx, const double *hy, const uint8_t *ht,
            long long nbond, const int32_t *hbond, dpd_cells &out) {
    if (!(L > 0) || !(cfg.h > 0) || !(cfg.r_tail > 0) || !(cfg.r_stamp >= 0) || n64 < 0 || nbond < 0)
        throw Fail{DPD_E_ARG, "cell detection: bad box, configuration or sizes"};
    if (n64 >= INT_MAX / 2 || nbond >= INT_MAX / 4) throw Fail{DPD_E_ARG, "cell detection: too many beads or bonds"};
    const int n = (int)n64;
    const int nbd = (int)nbond;
    for (long long e = 0; e < 2 * nbond; e++)
        if (hbond[e] < 0 || hbond[e] >= n) throw Fail{DPD_E_ARG, "cell detection: a bond index is out of range"};
    for (int i = 0; i < n; i++)
        if (!(hx[i] >= 0.0 && hx[i] < L && hy[i] >= 0.0 && hy[i] < L))
            throw Fail{DPD_E_ARG, "cell detection: a position is outside [0, L) (wrap the snapshot's positions)"};
    const long long ng = (long long)std::nearbyint(L / cfg.h);  // round half to even, as Python's round
    if (ng < 4 || ng > 21845) throw Fail{DPD_E_ARG, "cell detection: the label grid side L/h must be 4..21845"};
    const double h = L / (double)ng;
    const long long G = ng * ng;
    out.h = h;
    out.ng = ng;
    const double r_pix = cfg.r_stamp / h;
    std::vector<int2> hoffs;
    {
        const int R = (int)std::floor(r_pix);
        for (int di = -R; di <= R; di++)
            for (int dj = -R; dj <= R; dj++)
                if (std::sqrt((double)(di * di + dj * dj)) <= r_pix) hoffs.push_back(make_int2(di, dj));
    }
    const int noff = (int)hoffs.size();

    Ctx c;
    c.init();
    int *err = c.err;
    const double *X = c.upload(hx, n), *Y = c.upload(hy, n);
    const uint8_t *TY = c.upload(ht, n);
    const int *BD = c.upload(hbond, 2 * (size_t)nbond);
    const int2 *OFF = c.upload(hoffs);

    // ---- 1. molecules
    int *par = c.alloc<int>(n);
    c.each(n, [=] __device__(long long i) { par[i] = (TY[i] == TH || TY[i] == TT) ? (int)i : -1; });
    c.each(nbd, [=] __device__(long long e) {
        const int a = BD[2 * e], b = BD[2 * e + 1];
        const int ta = TY[a], tb = TY[b];
        if ((ta == TH || ta == TT) && (tb == TH || tb == TT)) uf_union(par, a, b, err);
    });
    int *flag = c.alloc<int>(std::max(n, 1));
    c.each(n, [=] __device__(long long i) { flag[i] = par[i] == (int)i; });
    int *rank = c.alloc<int>(std::max(n, 1));
    const int nmol = scan(c, flag, rank, (long long)n);
    int *mol = c.alloc<int>(n);
    c.each(n, [=] __device__(long long i) { mol[i] = par[i] < 0 ? -1 : rank[uf_find(par, (int)i)]; });
    c.check_flags("molecules");
    long long nlipid = 0;
    {
        std::vector<uint8_t> t(ht, ht + n);
        for (int i = 0; i < n; i++) nlipid += (t[i] == TH || t[i] == TT);
    }

    // ---- 2. tail contacts and aggregates
    int ncs = (int)std::floor(L / cfg.r_tail);
    if (ncs < 3) ncs = 1;
    const double cw = L / ncs;
    const long long NC = (long long)ncs * ncs;
    int *ccount = c.zeros<int>(NC + 1), *tcell = c.alloc<int>(n);
    c.each(n, [=] __device__(long long i) {
        if (TY[i] != TT) return;
        const int cx = min((int)(X[i] / cw), ncs - 1), cy = min((int)(Y[i] / cw), ncs - 1);
        tcell[i] = cx * ncs + cy;
        atomicAdd(ccount + tcell[i], 1);
    });
    int *cstart = c.alloc<int>(NC + 1);
    const int nT = scan(c, ccount, cstart, NC + 1);
    int *cur = c.alloc<int>(NC + 1), *tlist = c.alloc<int>(nT);
    CU(cudaMemcpyAsync(cur, cstart, (NC + 1) * sizeof(int), cudaMemcpyDeviceToDevice, c.s));
    c.each(n, [=] __device__(long long i) {
        if (TY[i] == TT) tlist[atomicAdd(cur + tcell[i], 1)] = (int)i;
    });
    const double r2t = cfg.r_tail * cfg.r_tail;
    const int rx = ncs >= 3 ? 1 : 0;
    // pairs (i, j), i < j, of T beads within r_tail: counted (pass 0), then written (pass 1)
    int *pcnt = c.zeros<int>(n), *poff = c.alloc<int>(n);
    int npair = 0;
    int2 *PR = nullptr;
    for (int pass = 0; pass < 2; pass++) {
        if (pass == 1) {
            npair = scan(c, pcnt, poff, (long long)n);
            PR = c.alloc<int2>(npair);
        }
        if (nmol == 0 || nT < 2 || (pass == 1 && npair == 0)) continue;
        int *cnt_out = pass == 0 ? pcnt : nullptr;
        const int *off = pass == 1 ? poff : nullptr;
        int2 *pairs = PR;
        c.each(n, [=] __device__(long long ii) {
            const int i = (int)ii;
            if (TY[i] != TT) return;
            const int cx = tcell[i] / ncs, cy = tcell[i] % ncs;
            int k = 0;
            const int o = off ? off[i] : 0;
            for (int ox = -rx; ox <= rx; ox++)
                for (int oy = -rx; oy <= rx; oy++) {
                    const int cc = ((cx + ox + ncs) % ncs) * ncs + (cy + oy + ncs) % ncs;
                    for (int q = cstart[cc]; q < cstart[cc + 1]; q++) {
                        const int j = tlist[q];
                        if (j <= i) continue;
                        const double dx = kd_wrap(__dsub_rn(X[j], X[i]), L), dy = kd_wrap(__dsub_rn(Y[j], Y[i]), L);
                        if (sq2(dx, dy) <= r2t) {
                            if (off) pairs[o + k] = make_int2(i, j);
                            k++;
                        }
                    }
                }
            if (cnt_out) cnt_out[i] = k;
        });
    }
    c.release(ccount);
    c.release(cur);
    c.release(pcnt);
    c.release(poff);

    int *par2 = c.alloc<int>(std::max(nmol, 1));
    c.each(nmol, [=] __device__(long long m) { par2[m] = (int)m; });
    c.each(npair, [=] __device__(long long e) { uf_union(par2, mol[PR[e].x], mol[PR[e].y], err); });
    c.each(nmol, [=] __device__(long long m) { flag[m] = par2[m] == (int)m; });
    const int nagg = scan(c, flag, rank, (long long)nmol);
    int *aggm = c.alloc<int>(std::max(nmol, 1)), *asz = c.zeros<int>(std::max(nagg, 1));
    c.each(nmol, [=] __device__(long long m) {
        aggm[m] = rank[uf_find(par2, (int)m)];
        atomicAdd(asz + aggm[m], 1);
    });
    int *bagg = c.alloc<int>(n);
    c.each(n, [=] __device__(long long i) { bagg[i] = mol[i] < 0 ? -1 : aggm[mol[i]]; });
    c.check_flags("aggregates");
    const std::vector<int> hasz = c.download(asz, nagg);

    long long n_free = 0, largest = 0;
    std::vector<int> cand;
    for (int a = 0; a < nagg; a++) {
        if (hasz[a] >= cfg.min_membrane_lipids)
            cand.push_back(a);
        else
            n_free += hasz[a];
        largest = std::max<long long>(largest, hasz[a]);
    }
    const int ncand = (int)cand.size();
    std::vector<uint8_t> hcand(std::max(nagg, 1), 0);
    for (int a : cand) hcand[a] = 1;
    const uint8_t *CAND = c.upload(hcand);

    // ---- 3. unwrapping: adjacency (out-neighbours then in-neighbours, each sorted, no repeats)
    int *dout = c.zeros<int>(n), *din = c.zeros<int>(n);
    auto edge_ok = [=] __device__(int a, int b) {
        return mol[a] >= 0 && mol[b] >= 0 && CAND[bagg[a]] != 0;
    };
    c.each(nbd, [=] __device__(long long e) {
        const int a = BD[2 * e], b = BD[2 * e + 1];
        if (!edge_ok(a, b)) return;
        atomicAdd(dout + a, 1);
        atomicAdd(din + b, 1);
    });
    c.each(npair, [=] __device__(long long e) {
        const int a = PR[e].x, b = PR[e].y;
        if (!CAND[bagg[a]]) return;
        atomicAdd(dout + a, 1);
        atomicAdd(din + b, 1);
    });
    int *dtot = c.alloc<int>(n), *aoff = c.alloc<int>(n);
    c.each(n, [=] __device__(long long i) { dtot[i] = dout[i] + din[i]; });
    const int nadj = scan(c, dtot, aoff, (long long)n);
    int *adj = c.alloc<int>(nadj), *co = c.zeros<int>(n), *ci = c.zeros<int>(n);
    c.each(nbd, [=] __device__(long long e) {
        const int a = BD[2 * e], b = BD[2 * e + 1];
        if (!edge_ok(a, b)) return;
        adj[aoff[a] + atomicAdd(co + a, 1)] = b;
        adj[aoff[b] + dout[b] + atomicAdd(ci + b, 1)] = a;
    });
    c.each(npair, [=] __device__(long long e) {
        const int a = PR[e].x, b = PR[e].y;
        if (!CAND[bagg[a]]) return;
        adj[aoff[a] + atomicAdd(co + a, 1)] = b;
        adj[aoff[b] + dout[b] + atomicAdd(ci + b, 1)] = a;
    });
    c.each(n, [=] __device__(long long i) {
        for (int part = 0; part < 2; part++) {
            int *s = adj + aoff[i] + (part ? dout[i] : 0);
            const int m = part ? din[i] : dout[i];
            for (int x = 1; x < m; x++) {  // insertion sort
                const int v = s[x];
                int y = x - 1;
                while (y >= 0 && s[y] > v) {
                    s[y + 1] = s[y];
                    y--;
                }
                s[y + 1] = v;
            }
            for (int x = m - 1; x > 0; x--)
                if (s[x] == s[x - 1]) s[x] = -1;  // repeated edge: kept once (the first)
        }
    });
    c.release(co);
    c.release(ci);

    // breadth-first walks from each membrane's lowest bead, all membranes at once
    int *rootmin = c.fill<int>(std::max(nagg, 1), 0x7f);
    c.each(n, [=] __device__(long long i) {
        if (mol[i] >= 0 && CAND[bagg[i]]) atomicMin(rootmin + bagg[i], (int)i);
    });
    const std::vector<int> hroot = c.download(rootmin, nagg);
    std::vector<int> f0;
    for (int a : cand) f0.push_back(hroot[a]);
    int *level = c.fill<int>(n, 0xff);
    unsigned long long *key = c.fill<unsigned long long>(n, 0xff);
    double *UX = c.alloc<double>(n), *UY = c.alloc<double>(n);
    int *F = c.alloc<int>(n), *Fn = c.alloc<int>(n), *C = c.alloc<int>(n), *O = c.alloc<int>(n);
    if (ncand) CU(cudaMemcpyAsync(F, f0.data(), ncand * sizeof(int), cudaMemcpyHostToDevice, c.s));
    CU(cudaStreamSynchronize(c.s));
    c.each(ncand, [=] __device__(long long k) {
        const int r = F[k];
        level[r] = 0;
        UX[r] = X[r];
        UY[r] = Y[r];
    });
    int nf = ncand;
    for (int d = 0; nf > 0; d++) {
        const int *Fc = F;
        c.each(nf, [=] __device__(long long k) {
            const int u = Fc[k];
            for (int s = 0; s < dtot[u]; s++) {
                const int v = adj[aoff[u] + s];
                if (v >= 0 && level[v] < 0) atomicMin(key + v, ((unsigned long long)k << 20) | (unsigned)s);
            }
        });
        c.each(nf, [=] __device__(long long k) {
            const int u = Fc[k];
            int m = 0;
            for (int s = 0; s < dtot[u]; s++) {
                const int v = adj[aoff[u] + s];
                if (v >= 0 && level[v] < 0 && key[v] == (((unsigned long long)k << 20) | (unsigned)s)) m++;
            }
            C[k] = m;
        });
        const int nn = scan(c, C, O, (long long)nf);
        int *Fo = Fn;
        c.each(nf, [=] __device__(long long k) {
            const int u = Fc[k];
            int j = O[k];
            for (int s = 0; s < dtot[u]; s++) {
                const int v = adj[aoff[u] + s];
                if (v >= 0 && level[v] < 0 && key[v] == (((unsigned long long)k << 20) | (unsigned)s)) {
                    Fo[j++] = v;
                    level[v] = d + 1;
                    UX[v] = __dadd_rn(UX[u], minimg(__dsub_rn(X[v], X[u]), L));
                    UY[v] = __dadd_rn(UY[u], minimg(__dsub_rn(Y[v], Y[u]), L));
                }
            }
        });
        std::swap(F, Fn);
        nf = nn;
    }
    c.release(key);
    c.release(C);
    c.release(O);
    c.release(F);
    c.release(Fn);

    // wrap test on every edge; bounding boxes of the unwrapped beads
    int *wr = c.zeros<int>(std::max(nagg, 1));
    auto wrap_edge = [=] __device__(int a, int b) {
        const double half = 0.5 * L;
        const double ex = __dsub_rn(__dsub_rn(UX[b], UX[a]), minimg(__dsub_rn(X[b], X[a]), L));
        const double ey = __dsub_rn(__dsub_rn(UY[b], UY[a]), minimg(__dsub_rn(Y[b], Y[a]), L));
        if (fabs(ex) > half || fabs(ey) > half) wr[bagg[a]] = 1;
    };
    c.each(nbd, [=] __device__(long long e) {
        const int a = BD[2 * e], b = BD[2 * e + 1];
        if (edge_ok(a, b)) wrap_edge(a, b);
    });
    c.each(npair, [=] __device__(long long e) {
        if (CAND[bagg[PR[e].x]]) wrap_edge(PR[e].x, PR[e].y);
    });
    unsigned long long *umin = c.fill<unsigned long long>(2 * (size_t)std::max(nagg, 1), 0xff);
    unsigned long long *umax = c.zeros<unsigned long long>(2 * (size_t)std::max(nagg, 1));
    c.each(n, [=] __device__(long long i) {
        if (mol[i] < 0 || !CAND[bagg[i]]) return;
        const int a = bagg[i];
        atomicMin(umin + 2 * a, dkey(UX[i]));
        atomicMin(umin + 2 * a + 1, dkey(UY[i]));
        atomicMax(umax + 2 * a, dkey(UX[i]));
        atomicMax(umax + 2 * a + 1, dkey(UY[i]));
    });
    std::vector<int> hwr = c.download(wr, nagg);
    const std::vector<unsigned long long> hmin = c.download(umin, 2 * (size_t)nagg), hmax = c.download(umax, 2 * (size_t)nagg);

    // ---- 4a. holes of the membranes that do not wrap: one box each
    struct Box {
        long long base, lo0, lo1;
        int s0, s1, agg;
    };
    std::vector<Box> boxes;
    std::vector<int> hboxof(std::max(nagg, 1), -1);
    long long P = 0;
    for (int a : cand) {
        if (hwr[a]) continue;
        const long long lo0 = (long long)std::floor((dkey_inv(hmin[2 * a]) - cfg.pad) / h);
        const long long lo1 = (long long)std::floor((dkey_inv(hmin[2 * a + 1]) - cfg.pad) / h);
        const long long hi0 = (long long)std::ceil((dkey_inv(hmax[2 * a]) + cfg.pad) / h);
        const long long hi1 = (long long)std::ceil((dkey_inv(hmax[2 * a + 1]) + cfg.pad) / h);
        const long long s0 = hi0 - lo0 + 1, s1 = hi1 - lo1 + 1;
        if (s0 * s1 > 9 * G) {  // absurdly large: treated as wrapping (cells.py:384-385)
            hwr[a] = 1;
            continue;
        }
        hboxof[a] = (int)boxes.size();
        boxes.push_back(Box{P, lo0, lo1, (int)s0, (int)s1, a});
        P += s0 * s1;
    }
    if (P >= INT_MAX) throw Fail{DPD_E_ARG, "cell detection: the membranes' bounding boxes exceed 2^31 pixels"};
    const int nbox = (int)boxes.size();
    const long long min_px = std::max<long long>(0, (long long)std::floor(cfg.min_lumen_area / (h * h)) - 1);
    std::vector<int> n_holes(std::max(nagg, 1), 0);
    // lumens per membrane, in the order cells.py lists its holes
    std::vector<std::vector<Lumen>> lum_of(std::max(nagg, 1));
    if (nbox) {
        std::vector<long long> hb(nbox + 1), hl0(nbox), hl1(nbox);
        std::vector<int> hs0(nbox), hs1(nbox);
        for (int b = 0; b < nbox; b++) {
            hb[b] = boxes[b].base;
            hl0[b] = boxes[b].lo0;
            hl1[b] = boxes[b].lo1;
            hs0[b] = boxes[b].s0;
            hs1[b] = boxes[b].s1;
        }
        hb[nbox] = P;
        const long long *BB = c.upload(hb), *BL0 = c.upload(hl0), *BL1 = c.upload(hl1);
        const int *BS0 = c.upload(hs0), *BS1 = c.upload(hs1), *BOXOF = c.upload(hboxof);
        const int Pi = (int)P;
        uint8_t *memb = c.zeros<uint8_t>(P);
        c.each(n, [=] __device__(long long i) {
            if (mol[i] < 0) return;
            const int b = BOXOF[bagg[i]];
            if (b < 0) return;
            const long long pi = (long long)floor(UX[i] / h) - BL0[b], pj = (long long)floor(UY[i] / h) - BL1[b];
            const int s0 = BS0[b], s1 = BS1[b];
            for (int o = 0; o < noff; o++) {
                const long long ii = pi + OFF[o].x, jj = pj + OFF[o].y;
                if (ii >= 0 && ii < s0 && jj >= 0 && jj < s1) memb[BB[b] + ii * s1 + jj] = 1;
            }
        });
        // every solvent pixel starts under the first pixel of its row run; a
        // vertical union is needed only where an overlap of two runs begins
        int *lp = c.alloc<int>(P), *rk = c.alloc<int>(P);
        c.each(Pi, [=] __device__(long long p) {
            const int b = find_seg(BB, nbox, p);
            const long long j = (p - BB[b]) % BS1[b];
            rk[p] = (memb[p] || j == 0 || memb[p - 1]) ? (int)p : -1;
        });
        max_scan(c, rk, lp, P);
        c.each(Pi, [=] __device__(long long p) {
            if (memb[p]) lp[p] = -1;
        });
        c.each(Pi, [=] __device__(long long p) {
            if (memb[p]) return;
            const int b = find_seg(BB, nbox, p);
            const long long loc = p - BB[b];
            const int s0 = BS0[b], s1 = BS1[b];
            const long long i = loc / s1, j = loc % s1;
            if (i + 1 < s0 && !memb[p + s1] && (j == 0 || memb[p - 1] || memb[p - 1 + s1]))
                uf_union(lp, (int)p, (int)(p + s1), err);
        });
        c.each(Pi, [=] __device__(long long p) {
            if (rk[p] == (int)p && !memb[p]) uf_flatten(lp, (int)p);
        });
        c.release(rk);
        int *sz = c.zeros<int>(P), *bord = c.zeros<int>(P);
        c.each(Pi, [=] __device__(long long p) {
            if (memb[p]) return;
            const int b = find_seg(BB, nbox, p);
            const long long loc = p - BB[b];
            const int s0 = BS0[b], s1 = BS1[b];
            const long long i = loc / s1, j = loc % s1;
            const int r = uf_find(lp, (int)p);
            agg_inc(sz, r);
            if (i == 0 || i == s0 - 1 || j == 0 || j == s1 - 1) bord[r] = 1;
        });
        c.check_flags("local holes");
        int *pf = c.alloc<int>(P);
        c.each(Pi, [=] __device__(long long p) { pf[p] = !memb[p] && lp[p] == (int)p && !bord[p]; });
        int *hroots = nullptr;
        const int nh = select_flags(c, pf, Pi, &hroots);
        int *hsz = c.alloc<int>(nh);
        c.each(nh, [=] __device__(long long k) { hsz[k] = sz[hroots[k]]; });
        const std::vector<int> hr = c.download(hroots, nh), hs = c.download(hsz, nh);
        std::vector<int> lroot, lsz, lagg;
        for (int k = 0; k < nh; k++) {
            const int b = (int)(std::upper_bound(hb.begin(), hb.end(), (long long)hr[k]) - hb.begin()) - 1;
            const int a = boxes[b].agg;
            n_holes[a]++;
            const double area = (double)hs[k] * h * h;
            if (area >= cfg.min_lumen_area) {
                lroot.push_back(hr[k]);
                lsz.push_back(hs[k]);
                lagg.push_back(a);
            }
        }
        const int nq = (int)lroot.size();
        if (nq) {
            int *lumid = c.fill<int>(P, 0xff);
            const int *LR = c.upload(lroot);
            c.each(nq, [=] __device__(long long q) { lumid[LR[q]] = (int)q; });
            c.each(Pi, [=] __device__(long long p) { pf[p] = !memb[p] && lumid[uf_find(lp, (int)p)] >= 0; });
            int *pix = nullptr;
            const int np_ = select_flags(c, pf, Pi, &pix);
            int *qk = c.alloc<int>(np_);
            c.each(np_, [=] __device__(long long e) { qk[e] = lumid[uf_find(lp, pix[e])]; });
            sort_pairs(c, qk, pix, np_, bits_for(nq));
            int2 *pool = c.alloc<int2>(np_);
            c.each(np_, [=] __device__(long long e) {
                const long long p = pix[e];
                const int b = find_seg(BB, nbox, p);
                const long long loc = p - BB[b];
                const int s1 = BS1[b];
                pool[e] = make_int2((int)(loc / s1 + BL0[b]), (int)(loc % s1 + BL1[b]));
            });
            long long o = 0;
            for (int q = 0; q < nq; q++) {
                lum_of[lagg[q]].push_back(Lumen{lagg[q], pool + o, lsz[q], (double)lsz[q] * h * h, false});
                o += lsz[q];
            }
            c.release(lumid);
            c.release(pix);
            c.release(qk);
        }
        c.release(memb);
        c.release(lp);
        c.release(sz);
        c.release(bord);
        c.release(pf);
        c.release(hroots);
        c.release(hsz);
    }

    // ---- 4b. holes of the wrapping membranes: the periodic grid, one membrane at a time
    for (int a : cand) {
        if (!hwr[a]) continue;
        const int Gi = (int)G;
        const long long ngl = ng;
        uint8_t *memb = c.zeros<uint8_t>(G);
        c.each(n, [=] __device__(long long i) {
            if (bagg[i] != a || mol[i] < 0) return;
            const long long pi = pmod((long long)floor(X[i] / h), ngl), pj = pmod((long long)floor(Y[i] / h), ngl);
            for (int o = 0; o < noff; o++) memb[pmod(pi + OFF[o].x, ngl) * ngl + pmod(pj + OFF[o].y, ngl)] = 1;
        });
        // row runs as in the boxes; unions (and the offset checks below) only on
        // the edges that leave a run: across the box edge along a row, and where
        // an overlap of two vertically adjacent runs begins.  Any other edge
        // closes a square of edges whose offsets are already consistent.
        unsigned long long *wp = c.alloc<unsigned long long>(G);
        int *rk = c.alloc<int>(G), *rs = c.alloc<int>(G);
        c.each(Gi, [=] __device__(long long p) {
            const long long j = p % ngl;
            rk[p] = (memb[p] || j == 0 || memb[p - 1]) ? (int)p : -1;
        });
        max_scan(c, rk, rs, G);
        c.each(Gi, [=] __device__(long long p) { wp[p] = memb[p] ? ~0ull : wpack(rs[p], 0, 0); });
        c.release(rk);
        c.release(rs);
        c.each(Gi, [=] __device__(long long p) {
            if (memb[p]) return;
            const long long i = p / ngl, j = p % ngl;
            if (j + 1 == ngl && !memb[i * ngl]) wunion(wp, (int)p, (int)(i * ngl), 0, 1, err);
            const long long q = (i + 1 == ngl ? 0 : i + 1) * ngl + j;
            if (!memb[q] && (j == 0 || memb[p - 1] || memb[q - 1])) wunion(wp, (int)p, (int)q, i + 1 == ngl ? 1 : 0, 0, err);
        });
        c.each(Gi, [=] __device__(long long p) {
            if (!memb[p] && (p % ngl == 0 || memb[p - 1])) wflatten(wp, (int)p);
        });
        int *wflag = c.zeros<int>(G), *cnt = c.zeros<int>(G);
        unsigned long long *si = c.zeros<unsigned long long>(G), *sj = c.zeros<unsigned long long>(G);
        c.each(Gi, [=] __device__(long long p) {
            if (memb[p]) return;
            const long long i = p / ngl, j = p % ngl;
            int ox, oy;
            const int r = wfind(wp, (int)p, ox, oy);
            const long long q[2] = {i * ngl + (j + 1 == ngl ? 0 : j + 1), (i + 1 == ngl ? 0 : i + 1) * ngl + j};
            const int sx[2] = {0, i + 1 == ngl ? 1 : 0}, sy[2] = {j + 1 == ngl ? 1 : 0, 0};
            for (int k = 0; k < 2; k++) {
                if (memb[q[k]]) continue;
                if (k == 0 && j + 1 != ngl) continue;                            // inside a run
                if (k == 1 && j != 0 && !memb[p - 1] && !memb[q[1] - 1]) continue;  // inside an overlap
                int qx, qy;
                const int rq = wfind(wp, (int)q[k], qx, qy);
                if (rq != r) atomicOr(err, 2);
                if (qx != ox + sx[k] || qy != oy + sy[k]) wflag[r] = 1;
            }
            agg_inc(cnt, r);
            atomicAdd(si + r, (unsigned long long)(i + (long long)ox * ngl));
            atomicAdd(sj + r, (unsigned long long)(j + (long long)oy * ngl));
        });
        c.check_flags("periodic holes");
        int *pf = c.alloc<int>(G);
        c.each(Gi, [=] __device__(long long p) { pf[p] = !memb[p] && wpar(wp[p]) == (int)p; });
        int *roots = nullptr;
        const int nr = select_flags(c, pf, Gi, &roots);
        int *rw = c.alloc<int>(nr), *rc = c.alloc<int>(nr);
        long long *rsi = c.alloc<long long>(nr), *rsj = c.alloc<long long>(nr);
        c.each(nr, [=] __device__(long long k) {
            const int r = roots[k];
            rw[k] = wflag[r];
            rc[k] = cnt[r];
            rsi[k] = (long long)si[r];
            rsj[k] = (long long)sj[r];
        });
        const std::vector<int> hr = c.download(roots, nr), hw = c.download(rw, nr), hc = c.download(rc, nr);
        const std::vector<long long> hsi = c.download(rsi, nr), hsj = c.download(rsj, nr);
        std::vector<int> tr, tsx, tsy;
        std::vector<long long> tcnt;
        for (int k = 0; k < nr; k++) {
            if (hw[k]) continue;
            n_holes[a]++;
            const long long m = hc[k];
            if (m < std::max<long long>(min_px, 1) || !((double)m * h * h >= cfg.min_lumen_area)) continue;
            // the copy whose centroid lies in the box (cells.py:280-292)
            const double dng = (double)ng;
            long long ssi = (long long)std::floor((double)hsi[k] / (double)m / dng);
            long long ssj = (long long)std::floor((double)hsj[k] / (double)m / dng);
            long long usi = ssi, usj = ssj;
            for (int it = 0; it < 4; it++) {
                usi = ssi;
                usj = ssj;
                const double ci = (double)(hsi[k] + (1 - ssi) * ng * m) / (double)m;
                const double cj = (double)(hsj[k] + (1 - ssj) * ng * m) / (double)m;
                const int di = ci < dng ? -1 : (ci >= 2 * dng ? 1 : 0);
                const int dj = cj < dng ? -1 : (cj >= 2 * dng ? 1 : 0);
                if (di == 0 && dj == 0) break;
                ssi += di;
                ssj += dj;
            }
            tr.push_back(hr[k]);
            tsx.push_back((int)usi);
            tsy.push_back((int)usj);
            tcnt.push_back(m);
        }
        const int nt = (int)tr.size();
        if (nt) {
            int *hid = c.fill<int>(G, 0xff);
            const int *TR = c.upload(tr), *TSX = c.upload(tsx), *TSY = c.upload(tsy);
            c.each(nt, [=] __device__(long long t) { hid[TR[t]] = (int)t; });
            c.each(Gi, [=] __device__(long long p) {
                int ox, oy;
                pf[p] = !memb[p] && hid[wfind(wp, (int)p, ox, oy)] >= 0;
            });
            int *pix = nullptr;
            const int np_ = select_flags(c, pf, Gi, &pix);
            unsigned long long *keys = c.alloc<unsigned long long>(np_);
            c.each(np_, [=] __device__(long long e) {
                const long long p = pix[e], i = p / ngl, j = p % ngl;
                int ox, oy;
                const int t = hid[wfind(wp, (int)p, ox, oy)];
                const long long fi = i + ((long long)ox - TSX[t]) * ngl + KEY_BIAS;
                const long long fj = j + ((long long)oy - TSY[t]) * ngl + KEY_BIAS;
                if (fi < 0 || fi >= 2 * KEY_BIAS || fj < 0 || fj >= 2 * KEY_BIAS) atomicOr(err, 4);
                keys[e] = ((unsigned long long)t << 40) | ((unsigned long long)fi << 20) | (unsigned long long)fj;
            });
            c.check_flags("periodic holes");
            sort_keys(c, keys, np_, 40 + bits_for(nt));
            int2 *pool = c.alloc<int2>(np_);
            c.each(np_, [=] __device__(long long e) {
                const unsigned long long k = keys[e];
                pool[e] = make_int2((int)((k >> 20) & 0xfffff) - KEY_BIAS, (int)(k & 0xfffff) - KEY_BIAS);
            });
            std::vector<long long> off(nt + 1, 0);
            for (int t = 0; t < nt; t++) off[t + 1] = off[t] + tcnt[t];
            std::vector<std::pair<std::pair<int, int>, int>> order;
            for (int t = 0; t < nt; t++) {
                const int2 f = c.get(pool + off[t]);
                order.push_back({{f.x, f.y}, t});
            }
            std::sort(order.begin(), order.end());
            for (auto &o : order) {
                const int t = o.second;
                lum_of[a].push_back(Lumen{a, pool + off[t], tcnt[t], (double)tcnt[t] * h * h, true});
            }
            c.release(hid);
            c.release(pix);
            c.release(keys);
        }
        c.release(memb);
        c.release(wp);
        c.release(wflag);
        c.release(cnt);
        c.release(si);
        c.release(sj);
        c.release(pf);
        c.release(roots);
        c.release(rw);
        c.release(rc);
        c.release(rsi);
        c.release(rsj);
    }

    // ---- 5. lumens: largest first (a stable sort, cells.py:406), painted in that order
    std::vector<Lumen> lumens;
    for (int a : cand)
        for (auto &l : lum_of[a]) lumens.push_back(l);
    std::stable_sort(lumens.begin(), lumens.end(), [](const Lumen &p, const Lumen &q) { return p.area_raw > q.area_raw; });
    const int nl = (int)lumens.size();
    std::vector<long long> hloff(nl + 1, 0);
    for (int k = 0; k < nl; k++) hloff[k + 1] = hloff[k] + lumens[k].cnt;
    const long long nent64 = hloff[nl];
    if (nent64 >= INT_MAX) throw Fail{DPD_E_ARG, "cell detection: lumens exceed 2^31 pixels"};
    const int nent = (int)nent64;
    int2 *LP = c.alloc<int2>(nent);
    const long long *LOFF = c.upload(hloff);
    {  // one gather of every lumen's pixel list, in the sorted order
        std::vector<unsigned long long> hsrc(std::max(nl, 1));
        for (int k = 0; k < nl; k++) hsrc[k] = (unsigned long long)(uintptr_t)lumens[k].src;
        const unsigned long long *SRC = c.upload(hsrc);
        c.each(nent, [=] __device__(long long e) {
            const int k = find_seg(LOFF, nl, e);
            LP[e] = ((const int2 *)(uintptr_t)SRC[k])[e - LOFF[k]];
        });
    }
    int *lid = c.alloc<int>(nent);
    c.each(nent, [=] __device__(long long e) { lid[e] = find_seg(LOFF, nl, e); });
    const long long ngl = ng;
    const int Gi = (int)G;
    int *label = c.fill<int>(G, 0xff);
    c.each(nent, [=] __device__(long long e) {
        atomicMax(label + pmod(LP[e].x, ngl) * ngl + pmod(LP[e].y, ngl), lid[e]);
    });
    int *gflat = c.alloc<int>(n);
    c.each(n, [=] __device__(long long i) {
        gflat[i] = (int)(pmod((long long)floor(X[i] / h), ngl) * ngl + pmod((long long)floor(Y[i] / h), ngl));
    });
    unsigned long long *counts = c.zeros<unsigned long long>(7 * (size_t)std::max(nl, 1));
    c.each(n, [=] __device__(long long i) {
        const int t = TY[i];
        if (!is_solvent_type(t)) return;
        const int l = label[gflat[i]];
        if (l >= 0) atomicAdd(counts + 7 * l + t, 1ull);
    });
    unsigned long long *apx = c.zeros<unsigned long long>(std::max(nl, 1));
    c.each(Gi, [=] __device__(long long p) {
        const int l = label[p];
        if (l >= 0) agg_inc(apx, l);
    });

    // bulk medium and the lumen tests (cells.py:420-459)
    const double mlen = nmol ? (double)nlipid / (double)nmol : 4.0;
    const double wall_max = 2.0 * mlen * 0.5 + cfg.wall_extra;
    const int Mpx = (int)std::ceil(wall_max / h) + 2;
    uint8_t *outside = c.zeros<uint8_t>(G);
    uint8_t *sel = c.zeros<uint8_t>(nent);
    double *dob = c.alloc<double>(nent);
    unsigned long long *lnb = c.zeros<unsigned long long>(std::max(nl, 1)), *lnout = c.zeros<unsigned long long>(std::max(nl, 1));
    unsigned long long *lnsel = c.zeros<unsigned long long>(std::max(nl, 1)), *lnclose = c.zeros<unsigned long long>(std::max(nl, 1));
    bool out_any = false;
    if (nl) {
        uint8_t *memb = c.zeros<uint8_t>(G);
        c.each(n, [=] __device__(long long i) {
            if (mol[i] < 0) return;
            const long long pi = gflat[i] / ngl, pj = gflat[i] % ngl;
            for (int o = 0; o < noff; o++) memb[pmod(pi + OFF[o].x, ngl) * ngl + pmod(pj + OFF[o].y, ngl)] = 1;
        });
        int *gp = c.alloc<int>(G), *rk = c.alloc<int>(G);
        c.each(Gi, [=] __device__(long long p) {
            const long long j = p % ngl;
            rk[p] = (memb[p] || j == 0 || memb[p - 1]) ? (int)p : -1;
        });
        max_scan(c, rk, gp, G);
        c.release(rk);
        c.each(Gi, [=] __device__(long long p) {
            if (memb[p]) gp[p] = -1;
        });
        c.each(Gi, [=] __device__(long long p) {
            if (memb[p]) return;
            const long long i = p / ngl, j = p % ngl;
            if (j + 1 == ngl && !memb[i * ngl]) uf_union(gp, (int)p, (int)(i * ngl), err);
            const long long q = (i + 1 == ngl ? 0 : i + 1) * ngl + j;
            if (!memb[q] && (j == 0 || memb[p - 1] || memb[q - 1])) uf_union(gp, (int)p, (int)q, err);
        });
        c.each(Gi, [=] __device__(long long p) {
            if (!memb[p] && (p % ngl == 0 || memb[p - 1])) uf_flatten(gp, (int)p);
        });
        int *garea = c.zeros<int>(G);
        c.each(Gi, [=] __device__(long long p) {
            if (!memb[p]) agg_inc(garea, uf_find(gp, (int)p));
        });
        c.check_flags("bulk medium");
        int *pf = c.alloc<int>(G);
        c.each(Gi, [=] __device__(long long p) { pf[p] = !memb[p] && gp[p] == (int)p; });
        int *roots = nullptr;
        const int nr = select_flags(c, pf, Gi, &roots);
        int *ra = c.alloc<int>(nr);
        c.each(nr, [=] __device__(long long k) { ra[k] = garea[roots[k]]; });
        const std::vector<int> hra = c.download(ra, nr);
        long long tot = 0, mx = 0;
        for (int v : hra) {
            tot += v;
            mx = std::max<long long>(mx, v);
        }
        std::vector<uint8_t> big(nr);
        for (int k = 0; k < nr; k++) big[k] = (hra[k] == mx) || ((double)hra[k] >= 0.25 * (double)tot);
        out_any = nr > 0;
        uint8_t *bigf = c.zeros<uint8_t>(G);
        const uint8_t *BIG = c.upload(big);
        c.each(nr, [=] __device__(long long k) { bigf[roots[k]] = BIG[k]; });
        c.each(Gi, [=] __device__(long long p) { outside[p] = !memb[p] && bigf[uf_find(gp, (int)p)]; });
        c.release(memb);
        c.release(gp);
        c.release(garea);
        c.release(pf);
        c.release(roots);
        c.release(ra);
        c.release(bigf);

        // boundary pixels (a 4-neighbour labelled otherwise), distance to the bulk medium
        c.each(nent, [=] __device__(long long e) {
            const int k = lid[e];
            const long long pi = pmod(LP[e].x, ngl), pj = pmod(LP[e].y, ngl);
            const bool b = label[pmod(pi + 1, ngl) * ngl + pj] != k || label[pmod(pi - 1, ngl) * ngl + pj] != k ||
                           label[pi * ngl + pmod(pj + 1, ngl)] != k || label[pi * ngl + pmod(pj - 1, ngl)] != k;
            sel[e] = b;
            if (b) atomicAdd(lnb + k, 1ull);
            if (outside[pi * ngl + pj]) atomicAdd(lnout + k, 1ull);
        });
        const bool oa = out_any;
        c.each(nent, [=] __device__(long long e) {
            const int k = lid[e];
            if (!sel[e] && lnb[k] != 0) return;
            sel[e] = 1;
            double d = INFINITY;
            if (oa) {
                const long long pi = pmod(LP[e].x, ngl), pj = pmod(LP[e].y, ngl);
                // rows and columns outward from the pixel, each scan stopped once
                // it cannot beat the nearest found so far
                long long best = LLONG_MAX;
                for (int ax = 0; ax <= Mpx && (long long)ax * ax < best; ax++)
                    for (int sx = 0; sx < (ax ? 2 : 1); sx++) {
                        const long long row = pmod(pi + (sx ? -ax : ax), ngl) * ngl;
                        for (int ay = 0; ay <= Mpx; ay++) {
                            const long long d2 = (long long)ax * ax + (long long)ay * ay;
                            if (d2 >= best) break;
                            if (outside[row + pmod(pj + ay, ngl)] || outside[row + pmod(pj - ay, ngl)]) best = d2;
                        }
                    }
                if (best != LLONG_MAX) d = sqrt((double)best) * h;
            }
            dob[e] = d;
            atomicAdd(lnsel + k, 1ull);
            if (d <= wall_max) atomicAdd(lnclose + k, 1ull);
        });
    }
    const std::vector<unsigned long long> hcnt = c.download(counts, 7 * (size_t)nl), hapx = c.download(apx, nl);
    const std::vector<unsigned long long> hnout = c.download(lnout, nl), hnsel = c.download(lnsel, nl),
                                          hnclose = c.download(lnclose, nl);
    std::vector<int> keep;
    std::vector<double> l_area(nl), l_exp(nl), l_wall(nl, INFINITY);
    for (int k = 0; k < nl; k++) {
        const double area = (double)hapx[k] * h * h;
        const unsigned long long *q = &hcnt[7 * (size_t)k];
        const double hyd = (double)(q[TW] + q[TN] + q[TKA] + q[TKB]);
        const bool is_bulk = (double)hnout[k] / (double)lumens[k].cnt > 0.2;
        l_area[k] = area;
        l_exp[k] = is_bulk ? 0.0 : (double)hnclose[k] / (double)hnsel[k];
        if (area >= cfg.min_lumen_area && hyd >= cfg.min_aqueous_frac * cfg.rho * area && l_exp[k] >= cfg.min_exposure)
            keep.push_back(k);
    }
    // median distance of the kept lumens' boundary (numpy's median)
    std::vector<double> hdob;
    std::vector<uint8_t> hsel;
    if (!keep.empty()) {
        hdob = c.download(dob, nent);
        hsel = c.download(sel, nent);
    }
    for (int k : keep) {
        const long long o = hloff[k], m = lumens[k].cnt;
        std::vector<double> v;
        bool fin = false;
        for (long long e = o; e < o + m; e++)
            if (hsel[e]) {
                v.push_back(hdob[e]);
                fin |= std::isfinite(hdob[e]);
            }
        if (!fin || v.empty()) continue;
        std::sort(v.begin(), v.end());
        const size_t z = v.size();
        l_wall[k] = z % 2 ? v[z / 2] : (v[z / 2 - 1] + v[z / 2]) / 2.0;
    }
    const int nk = (int)keep.size();
    std::vector<int> newid(std::max(nl, 1), -1);
    for (int j = 0; j < nk; j++) newid[keep[j]] = j;
    const int *NEWID = c.upload(newid);
    c.each(Gi, [=] __device__(long long p) {
        const int l = label[p];
        label[p] = l >= 0 ? NEWID[l] : -1;
    });
    int *bcell = c.fill<int>(n, 0xff);
    c.each(n, [=] __device__(long long i) {
        if (!is_solvent_type(TY[i])) return;
        const int l = label[gflat[i]];
        if (l >= 0) bcell[i] = l;
    });

    // ---- 6. wall lipids and leaflets (cells.py:470-537)
    std::vector<long long> n_lip(nk, 0), inner(nk, 0), outer(nk, 0);
    std::vector<int> agg_lumens_of(std::max(nagg, 1), 0);
    for (int k : keep) agg_lumens_of[lumens[k].agg]++;
    if (nk) {
        std::vector<uint8_t> hasc(std::max(nagg, 1), 0);
        std::vector<int> aggc(nk);
        for (int j = 0; j < nk; j++) {
            aggc[j] = lumens[keep[j]].agg;
            hasc[aggc[j]] = 1;
        }
        const uint8_t *HASC = c.upload(hasc);
        const int *AGGC = c.upload(aggc);
        const int BK = 8;
        const long long nbk = (ng + BK - 1) / BK;
        int *bc = c.zeros<int>(nbk * nbk + 1), *bo = c.alloc<int>(nbk * nbk + 1);
        c.each(nent, [=] __device__(long long e) {
            if (!sel[e] || NEWID[lid[e]] < 0) return;
            const long long pi = pmod(LP[e].x, ngl), pj = pmod(LP[e].y, ngl);
            atomicAdd(bc + (pi / BK) * nbk + pj / BK, 1);
        });
        const int nbe = scan(c, bc, bo, nbk * nbk + 1);
        int *bcur = c.alloc<int>(nbk * nbk + 1);
        CU(cudaMemcpyAsync(bcur, bo, (nbk * nbk + 1) * sizeof(int), cudaMemcpyDeviceToDevice, c.s));
        int3 *bent = c.alloc<int3>(nbe);
        c.each(nent, [=] __device__(long long e) {
            const int j = NEWID[lid[e]];
            if (!sel[e] || j < 0) return;
            const long long pi = pmod(LP[e].x, ngl), pj = pmod(LP[e].y, ngl);
            bent[atomicAdd(bcur + (pi / BK) * nbk + pj / BK, 1)] = make_int3(j, (int)pi, (int)pj);
        });
        const double rmax = std::max(wall_max, cfg.leaflet_max);
        const int rb = ((int)std::ceil(rmax / h) + 1) / BK + 2;
        const bool all_blocks = 2 * rb + 1 >= nbk;
        const int partial = ng % BK ? 1 : 0;
        double *bd = c.alloc<double>(n);
        int *bl = c.alloc<int>(n);
        c.each(n, [=] __device__(long long i) {
            if (mol[i] < 0 || !HASC[bagg[i]]) return;
            const int a = bagg[i];
            const long long bx = (gflat[i] / ngl) / BK, by = (gflat[i] % ngl) / BK;
            double best = INFINITY;
            int bj = -1;
            auto scan_block = [&](long long cx, long long cy) {
                const long long blk = cx * nbk + cy;
                for (int q = bo[blk]; q < bo[blk + 1]; q++) {
                    const int3 t = bent[q];
                    if (AGGC[t.x] != a) continue;
                    const double px = ((double)t.y + 0.5) * h, py = ((double)t.z + 0.5) * h;
                    const double d2 = sq2(kd_wrap(__dsub_rn(X[i], px), L), kd_wrap(__dsub_rn(Y[i], py), L));
                    if (d2 < best || (d2 == best && t.x < bj)) {  // a tie: the lower lumen
                        best = d2;
                        bj = t.x;
                    }
                }
            };
            if (all_blocks) {
                for (long long u = 0; u < nbk; u++)
                    for (long long v = 0; v < nbk; v++) scan_block(u, v);
            } else {
                // rings of blocks outward; every pixel of ring r lies more than (r - 1) BK
                // pixels away (one block less where the grid ends in a partial block), so
                // once that exceeds the nearest found, no nearer pixel and no tie remains
                for (int r = 0; r <= rb; r++) {
                    const int sure = r - 1 - partial;
                    if (sure > 0) {
                        const double dmin = (double)(sure * BK) * h;
                        if (dmin * dmin > best) break;
                    }
                    for (int dx = -r; dx <= r; dx++)
                        for (int dy = -r; dy <= r; dy++) {
                            if (max(abs(dx), abs(dy)) != r) continue;
                            scan_block(pmod(bx + dx, nbk), pmod(by + dy, nbk));
                        }
                }
            }
            bd[i] = bj >= 0 ? sqrt(best) : INFINITY;
            bl[i] = bj;
        });
        unsigned long long *mbest = c.fill<unsigned long long>(std::max(nmol, 1), 0xff);
        int *mwin = c.fill<int>(std::max(nmol, 1), 0x7f);
        c.each(n, [=] __device__(long long i) {
            if (mol[i] >= 0 && HASC[bagg[i]]) atomicMin(mbest + mol[i], (unsigned long long)__double_as_longlong(bd[i]));
        });
        c.each(n, [=] __device__(long long i) {
            if (mol[i] >= 0 && HASC[bagg[i]] && (unsigned long long)__double_as_longlong(bd[i]) == mbest[mol[i]])
                atomicMin(mwin + mol[i], (int)i);
        });
        int *molc = c.fill<int>(std::max(nmol, 1), 0xff);
        unsigned long long *nlip = c.zeros<unsigned long long>(nk), *inn = c.zeros<unsigned long long>(nk),
                           *outr = c.zeros<unsigned long long>(nk);
        const double lin = cfg.leaflet_in, lmax = cfg.leaflet_max;
        c.each(nmol, [=] __device__(long long m) {
            const int w = mwin[m];
            if (w == 0x7f7f7f7f) return;
            if (bd[w] <= wall_max && bl[w] >= 0) {
                molc[m] = bl[w];
                atomicAdd(nlip + bl[w], 1ull);
            }
        });
        c.each(n, [=] __device__(long long i) {
            if (mol[i] < 0 || !HASC[bagg[i]]) return;
            const int cc = molc[mol[i]];
            if (cc < 0) return;
            bcell[i] = -cc - 2;
            if (TY[i] != TH) return;
            const double d = bd[i];
            if (d <= lin)
                atomicAdd(inn + bl[i], 1ull);
            else if (d <= lmax)
                atomicAdd(outr + bl[i], 1ull);
        });
        const std::vector<unsigned long long> a1 = c.download(nlip, nk), a2 = c.download(inn, nk), a3 = c.download(outr, nk);
        for (int j = 0; j < nk; j++) {
            n_lip[j] = (long long)a1[j];
            inner[j] = (long long)a2[j];
            outer[j] = (long long)a3[j];
        }
    }

    // ---- 7. per cell: moments and hull of the lumen pixels; the bilayer test
    std::vector<double> rows;
    std::vector<int> final_id(std::max(nk, 1), -1);
    if (nk) {
        unsigned long long *mom = c.zeros<unsigned long long>(5 * (size_t)nk);
        int *rf = c.alloc<int>(nent);
        c.each(nent, [=] __device__(long long e) {
            const int k = lid[e], j = NEWID[k];
            rf[e] = 0;
            if (j < 0) return;
            const long long gi = LP[e].x, gj = LP[e].y;
            atomicAdd(mom + 5 * j, (unsigned long long)gi);
            atomicAdd(mom + 5 * j + 1, (unsigned long long)gj);
            atomicAdd(mom + 5 * j + 2, (unsigned long long)(gi * gi));
            atomicAdd(mom + 5 * j + 3, (unsigned long long)(gj * gj));
            atomicAdd(mom + 5 * j + 4, (unsigned long long)(gi * gj));
            const bool first = e == LOFF[k] || LP[e - 1].x != LP[e].x;
            const bool last = e == LOFF[k + 1] - 1 || LP[e + 1].x != LP[e].x;
            rf[e] = first || last;
        });
        int *ext = nullptr;
        const int nx = select_flags(c, rf, nent, &ext);
        int *exj = c.alloc<int>(nx);
        int2 *exp_ = c.alloc<int2>(nx);
        c.each(nx, [=] __device__(long long q) {
            exj[q] = NEWID[lid[ext[q]]];
            exp_[q] = LP[ext[q]];
        });
        const std::vector<int> hj = c.download(exj, nx);
        const std::vector<int2> hp = c.download(exp_, nx);
        const std::vector<unsigned long long> hm = c.download(mom, 5 * (size_t)nk);
        std::vector<std::vector<std::pair<long long, long long>>> pts(nk);
        for (int q = 0; q < nx; q++) pts[hj[q]].push_back({hp[q].x, hp[q].y});
        std::vector<int> kept2;
        const double lo_if = cfg.inner_frac_lo, hi_if = cfg.inner_frac_hi;
        for (int j = 0; j < nk; j++) {
            const long long tot = inner[j] + outer[j];
            const double f_in = (double)inner[j] / (double)std::max<long long>(tot, 1);
            if (tot >= 6 && lo_if <= f_in && f_in <= hi_if) kept2.push_back(j);
        }
        for (size_t f = 0; f < kept2.size(); f++) final_id[kept2[f]] = (int)f;
        for (int j : kept2) {
            const int k = keep[j];
            const Lumen &lu = lumens[k];
            const long long m = lu.cnt;
            const long long Si = (long long)hm[5 * j], Sj = (long long)hm[5 * j + 1];
            const long long Sii = (long long)hm[5 * j + 2], Sjj = (long long)hm[5 * j + 3], Sij = (long long)hm[5 * j + 4];
            const double cx = ((double)Si / (double)m + 0.5) * h, cy = ((double)Sj / (double)m + 0.5) * h;
            double vxx = 1, vyy = 1, vxy = 0;
            if (m > 2) {
                const __int128 cxx = (__int128)m * Sii - (__int128)Si * Si, cyy = (__int128)m * Sjj - (__int128)Sj * Sj;
                const __int128 cxy = (__int128)m * Sij - (__int128)Si * Sj;
                const double nn1 = (double)m * (double)(m - 1);
                vxx = h * h * (double)cxx / nn1;
                vyy = h * h * (double)cyy / nn1;
                vxy = h * h * (double)cxy / nn1;
            }
            const double mean = 0.5 * (vxx + vyy), dd = std::sqrt(0.25 * (vxx - vyy) * (vxx - vyy) + vxy * vxy);
            const double ev0 = mean - dd, ev1 = mean + dd;
            const long long a2 = hull_area2(pts[j]);
            const double vol = 0.5 * (double)a2 * h * h;
            const double solidity = a2 > 0 ? (double)m * h * h / std::max(vol, 1e-9) : 1.0;
            const unsigned long long *q = &hcnt[7 * (size_t)k];
            const double row[DPD_CELL_COLS] = {py_mod(cx, L),
                                               py_mod(cy, L),
                                               l_area[k],
                                               (double)n_lip[j],
                                               (double)q[TKA],
                                               (double)q[TKB],
                                               (double)q[TN],
                                               (double)q[TW],
                                               (double)q[TZ],
                                               (double)lu.agg,
                                               (double)agg_lumens_of[lu.agg],
                                               (double)hasz[lu.agg],
                                               (double)inner[j],
                                               (double)outer[j],
                                               std::sqrt(ev1 / std::max(ev0, 1e-9)),
                                               solidity,
                                               std::sqrt(ev1) * 4,
                                               lu.wraps ? 1.0 : 0.0,
                                               l_exp[k],
                                               l_wall[k]};
            rows.insert(rows.end(), row, row + DPD_CELL_COLS);
        }
        const int *FID = c.upload(final_id);
        c.each(Gi, [=] __device__(long long p) {
            const int l = label[p];
            label[p] = l >= 0 ? FID[l] : -1;
        });
        c.each(n, [=] __device__(long long i) {
            const int v = bcell[i];
            if (v >= 0)
                bcell[i] = FID[v];
            else if (v <= -2) {
                const int f = FID[-v - 2];
                bcell[i] = f >= 0 ? -f - 2 : -1;
            }
        });
    }
    c.check_flags("wall lipids");

    // ---- outputs
    out.summary[0] = nmol;
    out.summary[1] = nagg;
    out.summary[2] = ncand;
    out.summary[3] = n_free;
    out.summary[4] = nmol ? largest : 0;
    long long nwrap = 0;
    for (int a : cand) {
        out.aggs.insert(out.aggs.end(), {(int64_t)a, (int64_t)hasz[a], (int64_t)(hwr[a] != 0), (int64_t)n_holes[a]});
        nwrap += hwr[a] != 0;
    }
    out.summary[5] = nwrap;
    out.cells = rows;
    out.n = n;
    CU(cudaStreamSynchronize(c.s));
    for (void *p : {(void *)label, (void *)bcell, (void *)mol, (void *)bagg}) c.adopt(p);
    out.label = label;
    out.bead_cell = bcell;
    out.mol = mol;
    out.bead_agg = bagg;
}

}  // namespace dpd_cells_impl

extern "C" int dpd_cells_default(dpd_cells_cfg *cfg) {
    if (!cfg) return lib_error(DPD_E_ARG, "dpd_cells_default: null");
    std::memset(cfg, 0, sizeof *cfg);
    cfg->r_tail = 1.0;
    cfg->h = 0.25;
    cfg->r_stamp = 0.75;
    cfg->min_membrane_lipids = 12;
    cfg->min_lumen_area = 16.0;
    cfg->min_aqueous_frac = 0.30;
    cfg->rho = 3.0;
    cfg->pad = 2.5;
    cfg->leaflet_in = 1.5;
    cfg->leaflet_max = 6.0;
    cfg->min_exposure = 0.8;
    cfg->wall_extra = 4.0;
    cfg->inner_frac_lo = 0.2;
    cfg->inner_frac_hi = 0.62;
    return DPD_OK;
}

extern "C" int dpd_cells_detect(const dpd_cells_cfg *cfg, double L, int64_t n, const double *x, const double *y,
                                const uint8_t *type, int64_t nbond, const int32_t *bonds, dpd_cells **out) {
    if (!cfg || !out || (n > 0 && (!x || !y || !type)) || (nbond > 0 && !bonds))
        return lib_error(DPD_E_ARG, "dpd_cells_detect: null argument");
    *out = nullptr;
    dpd_cells *r = new dpd_cells();
    try {
        dpd_cells_impl::detect(*cfg, L, n, x, y, type, nbond, bonds, *r);
    } catch (const dpd_cells_impl::Fail &f) {
        delete r;
        return lib_error(f.code, f.msg.c_str());
    } catch (const std::exception &e) {
        delete r;
        return lib_error(DPD_E_NOMEM, e.what());
    }
    *out = r;
    return DPD_OK;
}

extern "C" int dpd_cells_info(const dpd_cells *c, int64_t *info, double *h) {
    if (!c || !info) return lib_error(DPD_E_ARG, "dpd_cells_info: null");
    for (int k = 0; k < 6; k++) info[k] = c->summary[k];
    info[6] = c->ng;
    info[7] = (int64_t)(c->cells.size() / DPD_CELL_COLS);
    info[8] = (int64_t)(c->aggs.size() / 4);
    if (h) *h = c->h;
    return DPD_OK;
}

extern "C" int dpd_cells_fetch(const dpd_cells *c, double *cells, int64_t *aggs, void *label, int32_t label_bytes,
                               int32_t *bead_cell, int32_t *mol, int32_t *bead_agg) {
    if (!c) return lib_error(DPD_E_ARG, "dpd_cells_fetch: null");
    if (label && label_bytes != 4 && label_bytes != 2) return lib_error(DPD_E_ARG, "dpd_cells_fetch: label_bytes must be 2 or 4");
    const int64_t ncell = (int64_t)(c->cells.size() / DPD_CELL_COLS);
    if (label && label_bytes == 2 && ncell >= 32767)
        return lib_error(DPD_E_ARG, "dpd_cells_fetch: 32767 or more cells need a 4-byte label grid");
    if (cells && !c->cells.empty()) std::memcpy(cells, c->cells.data(), c->cells.size() * sizeof(double));
    if (aggs && !c->aggs.empty()) std::memcpy(aggs, c->aggs.data(), c->aggs.size() * sizeof(int64_t));
    const long long G = c->ng * c->ng;
    if (label && G) {
        if (label_bytes == 4) {
            if (cudaMemcpy(label, c->label, G * sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
                return lib_error(DPD_E_CUDA, "dpd_cells_fetch: copy of the label grid failed");
        } else {
            int16_t *d = nullptr;
            if (cudaMalloc(&d, G * sizeof(int16_t)) != cudaSuccess) {
                cudaGetLastError();
                return lib_error(DPD_E_NOMEM, "dpd_cells_fetch: device allocation failed");
            }
            const int32_t *src = c->label;
            dpd_cells_impl::k_each<<<(unsigned)((G + dpd_cells_impl::TPB - 1) / dpd_cells_impl::TPB),
                                     dpd_cells_impl::TPB>>>(G, [=] __device__(long long p) { d[p] = (int16_t)src[p]; });
            const cudaError_t e = cudaMemcpy(label, d, G * sizeof(int16_t), cudaMemcpyDeviceToHost);
            cudaFree(d);
            if (e != cudaSuccess) return lib_error(DPD_E_CUDA, "dpd_cells_fetch: copy of the label grid failed");
        }
    }
    const int32_t *src[3] = {c->bead_cell, c->mol, c->bead_agg};
    int32_t *dst[3] = {bead_cell, mol, bead_agg};
    for (int k = 0; k < 3; k++)
        if (dst[k] && c->n && cudaMemcpy(dst[k], src[k], c->n * sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
            return lib_error(DPD_E_CUDA, "dpd_cells_fetch: copy of a per-bead array failed");
    return DPD_OK;
}

extern "C" void dpd_cells_free(dpd_cells *c) { delete c; }
