// dpd_analysis.cu -- analysis of a replica's configuration on the GPU: clusters
// of beads of one type and their neighbour fraction (the reference's
// `snapcheck.py tclust`, cel/engine/tests/snapcheck.py:122-144).
//
// Two beads of type t are joined when their distance is <= rcut (rcut <= 1,
// so the 3 x 3 cells around a bead hold every partner); the clusters are the
// connected components.  A lock-free union-find over the bead slots links the
// larger root under the smaller one with a compare-and-swap, so every cluster
// ends with its lowest slot as root whatever the order of the links; full
// path compression then gives each bead its root.  The neighbour counts are
// those of the reference: for every bead of type t, the beads of any type and
// of type t within 1.0 (self excluded).  Distances are FP64 from the FP32
// positions with the minimum image, as the reference computes them from its
// snapshot.
#include "dpd_device.cuh"

namespace {

__device__ __forceinline__ int uf_find(int *parent, int i) {
    // path halving; parents only ever decrease, so the walk ends at the root
    // within as many steps as there are beads (GID_MASK bounds that)
    for (int it = 0; it <= (int)GID_MASK; it++) {
        const int p = __ldcg(parent + i);
        if (p == i) return i;
        const int g = __ldcg(parent + p);
        if (g != p) atomicCAS(parent + i, p, g);
        i = g;
    }
    return i;
}

__device__ __forceinline__ void uf_union(int *parent, int a, int b, DevStatus *status) {
    for (int it = 0; it < 4096; it++) {
        a = uf_find(parent, a);
        b = uf_find(parent, b);
        if (a == b) return;
        const int lo = a < b ? a : b, hi = a < b ? b : a;
        if (atomicCAS(parent + hi, hi, lo) == hi) return;  // hi was still a root: linked
        a = lo;                                            // someone moved hi first: find again
        b = hi;
    }
    raise_flag(status, DPD_F_ANALYSIS);
}

__device__ __forceinline__ double min_image(double d, double L) { return d - L * rint(d / L); }

}  // namespace

// parent[i] = i for the beads of type t of the replica, -1 for the others
__global__ void __launch_bounds__(BEAD_TPB) k_uf_init(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                      const Chunk *__restrict__ ch, int rep_index, int t,
                                                      int *__restrict__ parent, int *__restrict__ size) {
    const Chunk c = ch[blockIdx.x];
    if (c.rep != rep_index) return;
    const int d = c.begin + (int)threadIdx.x;
    if (d >= c.end) return;
    parent[d] = (int)(b.tg[cur][d] >> TYPE_SHIFT) == t ? d : -1;
    size[d] = 0;
}

// joins each bead of type t with the type-t beads of higher slot within rcut,
// and counts its neighbours within 1.0 (all types; type t)
__global__ void __launch_bounds__(BEAD_TPB) k_uf_link(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                      const Chunk *__restrict__ ch, int rep_index, int t, double rcut,
                                                      int *__restrict__ parent, unsigned long long *__restrict__ acc) {
    const Chunk c = ch[blockIdx.x];
    if (c.rep != rep_index) return;
    const RepDev &R = reps[c.rep];
    const int d = c.begin + (int)threadIdx.x;
    unsigned long long n_all = 0, n_same = 0;
    if (d < c.end && parent[d] >= 0) {
        const float2 *__restrict__ pos = b.pos[cur];
        const float2 pi = pos[d];
        const double L = (double)R.L, r2c = rcut * rcut;
        const int32_t *cs = b.cstart + R.c0;
        int cx, cy;
        cell_xy(R, pi.x, pi.y, cx, cy);
        const int rx = R.ncx >= 3 ? 1 : 0, ry = R.ncy >= 3 ? 1 : 0;
        for (int ox = -rx; ox <= rx; ox++)
            for (int oy = -ry; oy <= ry; oy++) {
                const int nx = (cx + ox + R.ncx) % R.ncx, ny = (cy + oy + R.ncy) % R.ncy;
                const int cc = nx * R.ncy + ny;
                for (int j = cs[cc]; j < cs[cc + 1]; j++) {
                    if (j == d) continue;
                    const float2 pj = pos[j];
                    const double dx = min_image((double)pj.x - (double)pi.x, L);
                    const double dy = min_image((double)pj.y - (double)pi.y, L);
                    const double r2 = dx * dx + dy * dy;
                    if (r2 > 1.0) continue;
                    const bool same = (int)(b.tg[cur][j] >> TYPE_SHIFT) == t;
                    n_all++;
                    n_same += same;
                    if (same && j > d && r2 <= r2c) uf_union(parent, d, j, b.status);
                }
            }
    }
    n_all = warp_sum_ll((long long)n_all);
    n_same = warp_sum_ll((long long)n_same);
    if (lane_id() == 0 && n_all) {
        atomicAdd(acc + 0, n_all);
        atomicAdd(acc + 1, n_same);
    }
}

// each bead's root, and the bead counted in its cluster's size
__global__ void __launch_bounds__(BEAD_TPB) k_uf_label(const Chunk *__restrict__ ch, int rep_index,
                                                       int *__restrict__ parent, int *__restrict__ size) {
    const Chunk c = ch[blockIdx.x];
    if (c.rep != rep_index) return;
    const int d = c.begin + (int)threadIdx.x;
    if (d >= c.end || parent[d] < 0) return;
    const int r = uf_find(parent, d);
    atomicAdd(size + r, 1);
}

// per cluster root: the cluster count, the largest size and the sum of squared sizes
__global__ void __launch_bounds__(BEAD_TPB) k_uf_stats(const Chunk *__restrict__ ch, int rep_index,
                                                       const int *__restrict__ parent, const int *__restrict__ size,
                                                       unsigned long long *__restrict__ acc) {
    const Chunk c = ch[blockIdx.x];
    if (c.rep != rep_index) return;
    const int d = c.begin + (int)threadIdx.x;
    long long nc = 0, sq = 0, nb = 0;
    unsigned mx = 0;
    if (d < c.end && parent[d] == d) {
        const long long s = size[d];
        nc = 1;
        sq = s * s;
        nb = s;
        mx = (unsigned)s;
    }
    nc = warp_sum_ll(nc);
    sq = warp_sum_ll(sq);
    nb = warp_sum_ll(nb);
    mx = __reduce_max_sync(0xffffffffu, mx);
    if (lane_id() == 0 && nc) {
        atomicAdd(acc + 2, (unsigned long long)nc);
        atomicAdd(acc + 3, (unsigned long long)sq);
        atomicAdd(acc + 4, (unsigned long long)nb);
        atomicMax(acc + 5, (unsigned long long)mx);
    }
}

// ---------------------------------------------------------------- membrane aggregates

// The first two stages of the reference's cell detection (cel/tools/cells.py:
// lipid_molecules 68-86, detect 345-366): molecules are the components of the
// bonds between lipid beads (H, T), aggregates the components of the molecules
// joined by tail-tail contacts (T-T distance <= r_tail).  One union-find over
// the lipid beads takes both kinds of edges: the prev/next links (every bead of
// a molecule is linked in template order) and the T-T contacts.

__global__ void __launch_bounds__(BEAD_TPB) k_agg_init(Bufs b, int cur, const Chunk *__restrict__ ch, int rep_index,
                                                       int *__restrict__ parent, int *__restrict__ size,
                                                       int *__restrict__ minlab) {
    const Chunk c = ch[blockIdx.x];
    if (c.rep != rep_index) return;
    const int d = c.begin + (int)threadIdx.x;
    if (d >= c.end) return;
    const int t = (int)(b.tg[cur][d] >> TYPE_SHIFT);
    parent[d] = (t == 1 || t == 2) ? d : -1;
    size[d] = 0;
    minlab[d] = 0x7fffffff;
}

__global__ void __launch_bounds__(BEAD_TPB) k_agg_link(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                       const Chunk *__restrict__ ch, int rep_index, double r_tail,
                                                       int *__restrict__ parent) {
    const Chunk c = ch[blockIdx.x];
    if (c.rep != rep_index) return;
    const RepDev &R = reps[c.rep];
    const int d = c.begin + (int)threadIdx.x;
    if (d >= c.end || parent[d] < 0) return;
    const int nx = b.link[cur][d].y;
    if (nx >= 0 && parent[nx] >= 0) uf_union(parent, d, nx, b.status);
    if ((int)(b.tg[cur][d] >> TYPE_SHIFT) != 2) return;
    const float2 *__restrict__ pos = b.pos[cur];
    const float2 pi = pos[d];
    const double L = (double)R.L, r2c = r_tail * r_tail;
    const int32_t *cs = b.cstart + R.c0;
    int cx, cy;
    cell_xy(R, pi.x, pi.y, cx, cy);
    for (int ox = -1; ox <= 1; ox++)
        for (int oy = -1; oy <= 1; oy++) {
            const int gx = (cx + ox + R.ncx) % R.ncx, gy = (cy + oy + R.ncy) % R.ncy;
            const int cc = gx * R.ncy + gy;
            for (int j = cs[cc]; j < cs[cc + 1]; j++) {
                if (j <= d || (int)(b.tg[cur][j] >> TYPE_SHIFT) != 2) continue;
                const float2 pj = pos[j];
                const double dx = min_image((double)pj.x - (double)pi.x, L);
                const double dy = min_image((double)pj.y - (double)pi.y, L);
                if (dx * dx + dy * dy <= r2c) uf_union(parent, d, j, b.status);
            }
        }
}

// per lipid bead: its root; molecules (beads without prev) counted per aggregate;
// the aggregate's smallest gid
__global__ void __launch_bounds__(BEAD_TPB) k_agg_label(Bufs b, int cur, const Chunk *__restrict__ ch, int rep_index,
                                                        int *__restrict__ parent, int *__restrict__ size,
                                                        int *__restrict__ minlab) {
    const Chunk c = ch[blockIdx.x];
    if (c.rep != rep_index) return;
    const int d = c.begin + (int)threadIdx.x;
    if (d >= c.end || parent[d] < 0) return;
    const int r = uf_find(parent, d);
    if (b.link[cur][d].x < 0) atomicAdd(size + r, 1);
    atomicMin(minlab + r, (int)(b.tg[cur][d] & GID_MASK));
}

// per aggregate root: counts (acc[2] aggregates, [3] membranes, [4] molecules,
// [5] largest, [6] molecules in small aggregates); per bead (gid order) its
// aggregate's smallest gid, -1 for other beads
__global__ void __launch_bounds__(BEAD_TPB) k_agg_stats(Bufs b, int cur, const Chunk *__restrict__ ch, int rep_index,
                                                        int nrep_beads, int min_lipids, const int *__restrict__ parent,
                                                        const int *__restrict__ size, const int *__restrict__ minlab,
                                                        unsigned long long *__restrict__ acc, int32_t *out_label) {
    const Chunk c = ch[blockIdx.x];
    if (c.rep != rep_index) return;
    const int d = c.begin + (int)threadIdx.x;
    long long na = 0, nm = 0, nmol = 0, small = 0;
    unsigned mx = 0;
    if (d < c.end) {
        const int p = parent[d];
        const int g = (int)(b.tg[cur][d] & GID_MASK);
        if (out_label && g < nrep_beads) out_label[g] = p >= 0 ? __ldcg(minlab + uf_find((int *)parent, d)) : -1;
        if (p == d) {
            const int s = size[d];
            na = 1;
            nm = s >= min_lipids;
            nmol = s;
            small = s < min_lipids ? s : 0;
            mx = (unsigned)s;
        }
    }
    na = warp_sum_ll(na);
    nm = warp_sum_ll(nm);
    nmol = warp_sum_ll(nmol);
    small = warp_sum_ll(small);
    mx = __reduce_max_sync(0xffffffffu, mx);
    if (lane_id() == 0 && na) {
        atomicAdd(acc + 2, (unsigned long long)na);
        atomicAdd(acc + 3, (unsigned long long)nm);
        atomicAdd(acc + 4, (unsigned long long)nmol);
        atomicMax(acc + 5, (unsigned long long)mx);
        atomicAdd(acc + 6, (unsigned long long)small);
    }
}

void launch_aggregates(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, int rep_index, int n,
                       double r_tail, int min_lipids, int *parent, int *size, int *minlab, unsigned long long *acc,
                       int32_t *out_label, cudaStream_t s) {
    cudaMemsetAsync(acc, 0, 8 * sizeof(unsigned long long), s);
    k_agg_init<<<nbch, BEAD_TPB, 0, s>>>(b, cur, bch, rep_index, parent, size, minlab);
    k_agg_link<<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch, rep_index, r_tail, parent);
    k_agg_label<<<nbch, BEAD_TPB, 0, s>>>(b, cur, bch, rep_index, parent, size, minlab);
    k_agg_stats<<<nbch, BEAD_TPB, 0, s>>>(b, cur, bch, rep_index, n, min_lipids, parent, size, minlab, acc,
                                          out_label);
}

void launch_type_clusters(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, int rep_index, int t,
                          double rcut, int *parent, int *size, unsigned long long *acc, cudaStream_t s) {
    cudaMemsetAsync(acc, 0, 8 * sizeof(unsigned long long), s);
    k_uf_init<<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch, rep_index, t, parent, size);
    k_uf_link<<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch, rep_index, t, rcut, parent, acc);
    k_uf_label<<<nbch, BEAD_TPB, 0, s>>>(bch, rep_index, parent, size);
    k_uf_stats<<<nbch, BEAD_TPB, 0, s>>>(bch, rep_index, parent, size, acc);
}
