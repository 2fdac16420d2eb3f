// dpd_kernels.cu -- cell sort, integrator, pair + bond forces and observables (sm_100a).
//
// One step of the production path (dpd_step) is
//   k_scan1, k_scan2   exclusive scan of the per-cell counts of the NEXT positions
//   k_place            provisional slot of every bead: an atomic cursor per cell
//   k_cellfix          per cell: order its beads by old slot (stable sort), dest[]
//   k_permute          gather the old slots into the new order AND apply the
//                      Groot-Warren update (fused; oercel.c:2303-2334 + 832-933)
//   [chemistry]        dpd_chem.cu
//   k_forces           pair + bond forces of the new configuration; epilogue:
//                      cell of the next position and its atomic count
// so the bead state is read and written once per kernel and the sort keys for
// step n+1 come out of the force kernel of step n.
#include <algorithm>

#include "dpd_chem.cuh"

// ---------------------------------------------------------------- keys (prime / build_cells)

// RESORT: the sort before a catalyst check (launch_resort), which runs only if
// some replica is flagged; the other replicas are keyed by the positions of
// the previous buffer, the ones their slot order was sorted by, so their
// order does not change.
template <bool INTEG, bool RESORT>
__global__ void __launch_bounds__(BEAD_TPB) k_keys(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                   const Chunk *__restrict__ ch) {
    if (RESORT && !b.resort[0]) return;
    const Chunk c = ch[blockIdx.x];
    const RepDev &R = reps[c.rep];
    const int i = c.begin + (int)threadIdx.x;
    const bool act = i < c.end;
    uint32_t key = 0;
    if (act) {
        float2 p = b.pos[RESORT && !b.resort[1 + c.rep] ? cur ^ 1 : cur][i];
        if (INTEG) {
            const float2 v = b.vh[cur][i], f = b.f[cur][i];
            p.x = advance1(p.x, v.x, f.x, R.dt, R.dt2, R.L);
            p.y = advance1(p.y, v.y, f.y, R.dt, R.dt2, R.L);
        }
        int cx, cy;
        key = (uint32_t)(R.c0 + cell_xy(R, p.x, p.y, cx, cy));
    }
    count_key(b.count, key, act);
    if (act) b.key[i] = key;
}

// ---------------------------------------------------------------- scan of the cell counts

__device__ __forceinline__ int block_exclusive_scan(int v, int *total) {
    __shared__ int ws[SCAN_TPB / 32];
    const int lane = (int)lane_id(), w = (int)threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = lane < (SCAN_TPB / 32) ? ws[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < (SCAN_TPB / 32)) ws[lane] = s;
    }
    __syncthreads();
    const int before = w > 0 ? ws[w - 1] : 0;
    *total = ws[SCAN_TPB / 32 - 1];
    return before + x - v;
}

// block-local exclusive scan; counts are consumed and zeroed for the next step
// ZERO: the counts are consumed and zeroed here; without it they stay for
// k_place<true>, which consumes them as its placement cursors.
template <bool ZERO>
__global__ void __launch_bounds__(SCAN_TPB) k_scan1(uint32_t *__restrict__ count, int32_t *__restrict__ cstart,
                                                    int32_t *__restrict__ bsum, long long C,
                                                    long long *__restrict__ step, int step_inc,
                                                    DevStatus *__restrict__ status, const int32_t *__restrict__ gate) {
    pdl_begin();
    if (gate && !*gate) return;
    const long long base = (long long)blockIdx.x * SCAN_PER_BLOCK + (long long)threadIdx.x * SCAN_PER_THREAD;
    int v[SCAN_PER_THREAD];
    int s = 0;
    if (base + SCAN_PER_THREAD <= C) {
        const uint4 q = *reinterpret_cast<const uint4 *>(count + base);
        v[0] = (int)q.x;
        v[1] = (int)q.y;
        v[2] = (int)q.z;
        v[3] = (int)q.w;
        if (ZERO) *reinterpret_cast<uint4 *>(count + base) = make_uint4(0u, 0u, 0u, 0u);
    } else {
#pragma unroll
        for (int k = 0; k < SCAN_PER_THREAD; k++) {
            v[k] = base + k < C ? (int)count[base + k] : 0;
            if (ZERO && base + k < C) count[base + k] = 0u;
        }
    }
#pragma unroll
    for (int k = 0; k < SCAN_PER_THREAD; k++) s += v[k];
    int total;
    int ex = block_exclusive_scan(s, &total);
    if (base + SCAN_PER_THREAD <= C) {
        int4 o;
        o.x = ex;
        o.y = ex + v[0];
        o.z = o.y + v[1];
        o.w = o.z + v[2];
        *reinterpret_cast<int4 *>(cstart + base) = o;
    } else {
#pragma unroll
        for (int k = 0; k < SCAN_PER_THREAD; k++) {
            if (base + k < C) cstart[base + k] = ex;
            ex += v[k];
        }
    }
    if (threadIdx.x == 0) {
        bsum[blockIdx.x] = total;
        if (step_inc && blockIdx.x == 0) {
            *step += 1;
            status->n_grow = 0u;  // the chemistry candidate lists of the new step start empty
            status->n_bond = 0u;
        }
    }
}

// add the totals of all earlier blocks; the last block writes cstart[C]
__global__ void __launch_bounds__(SCAN_TPB) k_scan2(int32_t *__restrict__ cstart, uint32_t *__restrict__ fill,
                                                    const int32_t *__restrict__ bsum, long long C, int nblocks,
                                                    const int32_t *__restrict__ gate) {
    pdl_begin();
    if (gate && !*gate) return;
    __shared__ int red[SCAN_TPB / 32];
    int part = 0;
    for (int k = (int)threadIdx.x; k < (int)blockIdx.x; k += SCAN_TPB) part += bsum[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
    if (lane_id() == 0) red[threadIdx.x >> 5] = part;
    __syncthreads();
    int prefix = 0;
#pragma unroll
    for (int w = 0; w < SCAN_TPB / 32; w++) prefix += red[w];
    const long long base = (long long)blockIdx.x * SCAN_PER_BLOCK + (long long)threadIdx.x * SCAN_PER_THREAD;
    if (base + SCAN_PER_THREAD <= C) {
        int4 o = *reinterpret_cast<const int4 *>(cstart + base);
        o.x += prefix;
        o.y += prefix;
        o.z += prefix;
        o.w += prefix;
        if (prefix != 0) *reinterpret_cast<int4 *>(cstart + base) = o;
        *reinterpret_cast<int4 *>(fill + base) = o;
    } else {
#pragma unroll
        for (int k = 0; k < SCAN_PER_THREAD; k++)
            if (base + k < C) {
                cstart[base + k] += prefix;
                fill[base + k] = (uint32_t)cstart[base + k];
            }
    }
    if ((int)blockIdx.x == nblocks - 1 && threadIdx.x == 0) cstart[C] = prefix + bsum[nblocks - 1];
}

// Single pass (decoupled look-back, after Merrill and Garland's single-pass
// prefix scan): a block scans its 1024 counts, publishes its total, then sums
// its predecessors' published values, stopping at the first inclusive prefix.
// Blocks take their index from a ticket counter that is never reset, so a
// block waits only on blocks that are already running, and the launch's epoch
// (ticket / blocks) tags every published word: words of earlier launches read
// as not yet published, and nothing has to be cleared between launches.
// Published word: epoch (30 bits) | flag (2 bits: 1 block total, 2 inclusive
// prefix) | value (32 bits).  Waits on a predecessor are bounded; a block that
// gives up raises DPD_F_WAIT.
#define LB_AGG 1ull
#define LB_INC 2ull
#define LB_SPIN_LIMIT (1 << 22)

__device__ __forceinline__ unsigned long long lb_load(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void lb_store(unsigned long long *p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__global__ void __launch_bounds__(SCAN_TPB) k_scan_lb(uint32_t *__restrict__ count, int32_t *__restrict__ cstart,
                                                      uint32_t *__restrict__ fill, unsigned long long *state,
                                                      unsigned long long *ticket, long long C, int nblocks,
                                                      long long *__restrict__ step, int step_inc,
                                                      DevStatus *__restrict__ status) {
    pdl_begin();
    __shared__ unsigned long long sh_ticket;
    __shared__ int sh_excl;
    if (threadIdx.x == 0) sh_ticket = atomicAdd(ticket, 1ull);
    __syncthreads();
    const int id = (int)(sh_ticket % (unsigned long long)nblocks);
    const unsigned long long epoch = (sh_ticket / (unsigned long long)nblocks) & 0x3FFFFFFFull;
    const long long base = (long long)id * SCAN_PER_BLOCK + (long long)threadIdx.x * SCAN_PER_THREAD;
    int v[SCAN_PER_THREAD];
    int sum = 0;
    if (base + SCAN_PER_THREAD <= C) {
        const uint4 q = *reinterpret_cast<const uint4 *>(count + base);
        v[0] = (int)q.x;
        v[1] = (int)q.y;
        v[2] = (int)q.z;
        v[3] = (int)q.w;
        *reinterpret_cast<uint4 *>(count + base) = make_uint4(0u, 0u, 0u, 0u);
    } else {
#pragma unroll
        for (int k = 0; k < SCAN_PER_THREAD; k++) {
            v[k] = base + k < C ? (int)count[base + k] : 0;
            if (base + k < C) count[base + k] = 0u;
        }
    }
#pragma unroll
    for (int k = 0; k < SCAN_PER_THREAD; k++) sum += v[k];
    int total;
    int ex = block_exclusive_scan(sum, &total);
    // publish this block's total, then find the sum of all earlier blocks
    if (threadIdx.x == 0) {
        lb_store(state + id, epoch << 34 | (id == 0 ? LB_INC : LB_AGG) << 32 | (unsigned)total);
        if (step_inc && id == 0) {
            *step += 1;
            status->n_grow = 0u;  // the chemistry candidate lists of the new step start empty
            status->n_bond = 0u;
        }
    }
    if (threadIdx.x < 32) {
        const int lane = (int)threadIdx.x;
        int excl = 0;
        bool gave_up = false;
        for (int j = id - 1; j >= 0;) {
            // lane k looks at block j - k; wait until each of them has published in this launch
            const int jj = j - lane;
            unsigned long long w = 0;
            if (jj >= 0) {
                int spins = 0;
                while (true) {
                    w = lb_load(state + jj);
                    if ((w >> 34) == epoch && ((w >> 32) & 3ull) != 0ull) break;
                    if (++spins > LB_SPIN_LIMIT) {
                        gave_up = true;
                        w = epoch << 34 | LB_INC << 32;  // stop here: the result is flagged as invalid
                        break;
                    }
                }
            }
            const bool inc = jj >= 0 && ((w >> 32) & 3ull) == LB_INC;
            const unsigned incm = __ballot_sync(0xffffffffu, inc);
            const int stop = incm ? __ffs(incm) - 1 : 31;  // the nearest inclusive prefix ends the walk
            int val = (jj >= 0 && lane <= stop) ? (int)(unsigned)(w & 0xFFFFFFFFull) : 0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
            excl += val;
            if (incm) break;
            j -= 32;
        }
        if (__any_sync(0xffffffffu, gave_up) && lane == 0) raise_flag(status, DPD_F_WAIT);
        if (lane == 0) {
            sh_excl = excl;
            if (id > 0) lb_store(state + id, epoch << 34 | LB_INC << 32 | (unsigned)(excl + total));
        }
    }
    __syncthreads();
    const int prefix = sh_excl;
    ex += prefix;
    if (base + SCAN_PER_THREAD <= C) {
        int4 o;
        o.x = ex;
        o.y = ex + v[0];
        o.z = o.y + v[1];
        o.w = o.z + v[2];
        *reinterpret_cast<int4 *>(cstart + base) = o;
        *reinterpret_cast<int4 *>(fill + base) = o;
    } else {
#pragma unroll
        for (int k = 0; k < SCAN_PER_THREAD; k++) {
            if (base + k < C) {
                cstart[base + k] = ex;
                fill[base + k] = (uint32_t)ex;
            }
            ex += v[k];
        }
    }
    if (id == nblocks - 1 && threadIdx.x == 0) cstart[C] = prefix + total;
}

// ---------------------------------------------------------------- placement and the stable fix-up

// The beads of a warp that go to the same cell share one atomic on its cursor
// and take consecutive places in lane (= old slot) order.
#ifndef PLACE_ITEMS
#define PLACE_ITEMS 4
#endif

// The sort without the second scan pass (sort_mode 2): k_scan1<false> leaves
// each cell's start within its scan block in `fill` and the counts in place;
// k_place<true> and k_cellfix<true> add the block prefixes themselves (every
// CTA scans the block totals into shared memory), k_place<true> takes the
// places by counting each cell's count down to zero (so the counts are clear
// for the next step's force epilogue), and k_cellfix<true> writes the final
// cell starts.
#define PFX_MAX 4096  // scan blocks whose prefixes a CTA holds: C <= 4,194,304 cells

// exclusive prefix of the scan's block totals, into shared memory (blockDim = SCAN_TPB)
__device__ __forceinline__ void block_prefixes(const int32_t *__restrict__ bsum, int nb, int *pfx) {
    const int per = (nb + SCAN_TPB - 1) / SCAN_TPB;
    const int lo = (int)threadIdx.x * per, hi = min(lo + per, nb);
    int s = 0;
    for (int k = lo; k < hi; k++) s += bsum[k];
    int total;
    int ex = block_exclusive_scan(s, &total);
    for (int k = lo; k < hi; k++) {
        pfx[k] = ex;
        ex += bsum[k];
    }
    __syncthreads();
}

// PLACE_ITEMS chunks per CTA: all keys are loaded before the first atomic
template <bool PFX>
__global__ void __launch_bounds__(BEAD_TPB) k_place(Bufs b, const Chunk *__restrict__ ch, int nch,
                                                    const int32_t *__restrict__ gate, int nb) {
    pdl_begin();
    if (gate && !*gate) return;
    __shared__ int pfx[PFX ? PFX_MAX : 1];
    if (PFX) block_prefixes(b.bsum, nb, pfx);
    const unsigned lane = lane_id();
    uint32_t key[PLACE_ITEMS];
    int idx[PLACE_ITEMS];
#pragma unroll
    for (int k = 0; k < PLACE_ITEMS; k++) {
        const int c = (int)blockIdx.x * PLACE_ITEMS + k;
        idx[k] = -1;
        if (c < nch) {
            const Chunk q = ch[c];
            const int i = q.begin + (int)threadIdx.x;
            if (i < q.end) idx[k] = i;
        }
        key[k] = idx[k] >= 0 ? b.key[idx[k]] : 0xFFFFFFFFu;
    }
#pragma unroll
    for (int k = 0; k < PLACE_ITEMS; k++) {
        const bool act = idx[k] >= 0;
        const unsigned grp = __match_any_sync(0xffffffffu, key[k]);
        const int leader = __ffs(grp) - 1;
        uint32_t base = 0;
        if (act && (int)lane == leader) {
            if (PFX) {
                const unsigned n = (unsigned)__popc(grp), left = atomicSub(b.count + key[k], n);
                base = b.fill[key[k]] + (uint32_t)pfx[key[k] / SCAN_PER_BLOCK] + left - n;
            } else {
                base = atomicAdd(b.fill + key[k], (unsigned)__popc(grp));
            }
        }
        base = __shfl_sync(0xffffffffu, base, leader);
        if (act) b.src[base + __popc(grp & ((1u << lane) - 1u))] = idx[k];
    }
}

// bitonic sort of NP register values (static indexing only)
template <int NP>
__device__ __forceinline__ void bitonic(int (&v)[NP]) {
#pragma unroll
    for (int k = 2; k <= NP; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1)
#pragma unroll
            for (int i = 0; i < NP; i++) {
                const int l = i ^ j;
                if (l > i) {
                    const bool up = (i & k) == 0;
                    const int a = v[i], c = v[l];
                    const bool sw = up ? (a > c) : (a < c);
                    v[i] = sw ? c : a;
                    v[l] = sw ? a : c;
                }
            }
}

template <int NP>
__device__ __forceinline__ void fix_cell(int32_t *__restrict__ src, int32_t *__restrict__ dest, int s, int m) {
    int v[NP];
    bool sorted = true;
#pragma unroll
    for (int k = 0; k < NP; k++) {
        v[k] = k < m ? src[s + k] : 0x7fffffff;
        if (k > 0) sorted = sorted && v[k - 1] <= v[k];
    }
    if (!sorted) bitonic<NP>(v);
#pragma unroll
    for (int k = 0; k < NP; k++)
        if (k < m) {
            if (!sorted) src[s + k] = v[k];
            dest[v[k]] = s + k;
        }
}

// Beads that land in one cell keep their old slot order (the reference's
// stable counting sort, oercel.c:832-933): the atomics gave each bead some
// place in its cell; here every cell orders its beads by old slot.
__device__ __forceinline__ void cellfix_range(const Bufs &b, int s, int m) {
    if (m <= 1) {
        if (m == 1) b.dest[b.src[s]] = s;
        return;
    }
    if (m <= 4) {
        fix_cell<4>(b.src, b.dest, s, m);
    } else if (m <= 8) {
        fix_cell<8>(b.src, b.dest, s, m);
    } else if (m <= 16) {
        fix_cell<16>(b.src, b.dest, s, m);
    } else {
        // crowded cell: in-place insertion sort in global memory
        atomicMax(&b.status->bigcell, (unsigned)m);
        for (int k = 1; k < m; k++) {
            const int t = b.src[s + k];
            int q = k - 1;
            while (q >= 0 && b.src[s + q] > t) {
                b.src[s + q + 1] = b.src[s + q];
                q--;
            }
            b.src[s + q + 1] = t;
        }
        for (int k = 0; k < m; k++) b.dest[b.src[s + k]] = s + k;
    }
}

template <bool PFX>
__global__ void __launch_bounds__(CELL_TPB) k_cellfix(Bufs b, const Chunk *__restrict__ ch,
                                                      const int32_t *__restrict__ gate, int nb, long long C) {
    pdl_begin();
    if (gate && !*gate) return;
    __shared__ int pfx[PFX ? PFX_MAX : 1];
    if (PFX) block_prefixes(b.bsum, nb, pfx);
    const Chunk c = ch[blockIdx.x];
    const int cell = c.begin + (int)threadIdx.x;
    if (cell >= c.end) return;
    int s, e;
    if (PFX) {  // the final cell starts: block-local start + block prefix
        s = (int)b.fill[cell] + pfx[cell / SCAN_PER_BLOCK];
        e = cell + 1 < C ? (int)b.fill[cell + 1] + pfx[(cell + 1) / SCAN_PER_BLOCK] : pfx[nb - 1] + b.bsum[nb - 1];
        b.cstart[cell] = s;
        if (cell + 1 == C) b.cstart[C] = e;
    } else {
        s = b.cstart[cell];
        e = b.cstart[cell + 1];
    }
    cellfix_range(b, s, e - s);
}

// ---------------------------------------------------------------- permute (+ integrate)

#define OBS_ITEMS 4  // chunks per round of k_observables

#ifndef PERM_ITEMS
#define PERM_ITEMS 1
#endif

// new slot d takes old bead src[d].  PERM_STEP applies the Groot-Warren update
// on the way (x += dt vh + dt^2 f; vt = vh + (1/2 + lambda) dt f; vh += dt f);
// PERM_KEEP applies it with every bead kept in its slot (the order and cell
// index of the last sort stay valid for a catalyst check that follows);
// PERM_PRIME takes the loaded velocity as the full velocity (vt = v);
// PERM_SORT moves everything unchanged.
// ITEMS chunks per CTA, one bead of each per thread; the loads of all items
// are issued phase by phase (slots, state, partner slots) so that each thread
// has several independent gathers in flight.  The gathers wait on memory
// (three dependent loads: slot, state, partner slots), so the kernel is held
// to 32 registers for 8 CTAs (all 64 warps) per SM: 24.6 us a step on the
// 1,048,576-bead box against 26.7 us at 6 CTAs; 2 or 4 ITEMS were slower
// (29.7, 39.9 us).
template <int MODE, int ITEMS>
__global__ void __launch_bounds__(BEAD_TPB, 8) k_permute(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                      const Chunk *__restrict__ ch, int nch,
                                                      const int32_t *__restrict__ gate) {
    pdl_begin();
    if (gate && !*gate) return;
    constexpr bool STEP = MODE == PERM_STEP || MODE == PERM_KEEP, KEEP = MODE == PERM_KEEP;
    const int nxt = cur ^ 1;
    const int32_t *__restrict__ src = b.src;
    const int32_t *__restrict__ dest = b.dest;
    const float2 *__restrict__ pos0 = b.pos[cur];
    const float2 *__restrict__ vh0 = b.vh[cur];
    const float2 *__restrict__ f0 = b.f[cur];
    const uint32_t *__restrict__ tg0 = b.tg[cur];
    const int2 *__restrict__ lk0 = b.link[cur];
    int d[ITEMS], i[ITEMS], rep[ITEMS];
    bool act[ITEMS];
#pragma unroll
    for (int k = 0; k < ITEMS; k++) {
        const int c = (int)blockIdx.x * ITEMS + k;
        act[k] = false;
        d[k] = 0;
        rep[k] = 0;
        if (c < nch) {
            const Chunk q = ch[c];
            d[k] = q.begin + (int)threadIdx.x;
            rep[k] = q.rep;
            act[k] = d[k] < q.end;
        }
    }
#pragma unroll
    for (int k = 0; k < ITEMS; k++) i[k] = act[k] ? (KEEP ? d[k] : src[d[k]]) : 0;
    float2 p[ITEMS], vh[ITEMS], f[ITEMS];
    uint32_t tg[ITEMS];
    int2 lk[ITEMS];
#pragma unroll
    for (int k = 0; k < ITEMS; k++) {
        if (!act[k]) continue;
        p[k] = pos0[i[k]];
        vh[k] = vh0[i[k]];
        tg[k] = tg0[i[k]];
        lk[k] = lk0[i[k]];
        f[k] = MODE == PERM_PRIME ? make_float2(0.0f, 0.0f) : f0[i[k]];
    }
    int2 nl[ITEMS];
#pragma unroll
    for (int k = 0; k < ITEMS; k++)
        if (act[k])
            nl[k] = KEEP ? lk[k] : make_int2(lk[k].x >= 0 ? dest[lk[k].x] : -1, lk[k].y >= 0 ? dest[lk[k].y] : -1);
    const long long step = STEP ? *b.step : 0;
#pragma unroll
    for (int k = 0; k < ITEMS; k++) {
        // the replica's sum of stirring terms at the new positions (warp sums, one atomic per warp)
        const RepDev &Rk = reps[rep[k]];
        if (Rk.stir_A != 0.0f) {  // uniform over the warp: its lanes share one chunk
            long long st = 0;
            if (act[k]) {
                float yn = p[k].y;
                if (STEP) yn = advance1(yn, vh[k].y, f[k].y, Rk.dt, Rk.dt2, Rk.L);
                st = stir_fix(Rk, yn);
            }
            st = warp_sum_ll(st);
            if (lane_id() == 0 && st != 0) atomicAdd((unsigned long long *)(b.stir + rep[k]), (unsigned long long)st);
        }
        if (!act[k]) continue;
        const int dd = d[k];
        float2 q = p[k], v = vh[k];
        if (STEP) {
            const RepDev &R = reps[rep[k]];
            const float2 ff = f[k];
            // the catalyst check uses the cell index of the last sort while every
            // bead moved less than 0.5; otherwise its replica is sorted first
            if (KEEP && cat_due(R, step) &&
                fmaxf(fabsf(__fmaf_rn(R.dt2, ff.x, R.dt * v.x)), fabsf(__fmaf_rn(R.dt2, ff.y, R.dt * v.y))) >= 0.5f) {
                b.resort[0] = 1;
                b.resort[1 + rep[k]] = 1;
            }
            q = make_float2(advance1(q.x, v.x, ff.x, R.dt, R.dt2, R.L), advance1(q.y, v.y, ff.y, R.dt, R.dt2, R.L));
            if (!(q.x >= 0.0f && q.x < R.L && q.y >= 0.0f && q.y < R.L)) raise_flag(b.status, DPD_F_OUTSIDE);
            b.vt[nxt][dd] = make_float2(__fmaf_rn(R.cvt, ff.x, v.x), __fmaf_rn(R.cvt, ff.y, v.y));
            v = make_float2(__fmaf_rn(R.dt, ff.x, v.x), __fmaf_rn(R.dt, ff.y, v.y));
            if (chem_due(R, step)) chem_in_permute(b, cur, R, step, rep[k], dd, q, tg[k], lk[k], nl[k]);
        } else if (MODE == PERM_PRIME) {
            b.vt[nxt][dd] = v;
        } else {
            b.vt[nxt][dd] = b.vt[cur][i[k]];
            b.f[nxt][dd] = f[k];
        }
        b.pos[nxt][dd] = q;
        b.vh[nxt][dd] = v;
        b.tg[nxt][dd] = tg[k];
        b.link[nxt][dd] = nl[k];
    }
}

// ---------------------------------------------------------------- pair + bond forces

#define MAXHIT 32

// Per bead d: F_d = sum_j w [a_ij - gamma w (rhat . vt_ij) + sigma theta_ij / sqrt(dt)] rhat
// over the 3x3 neighbour cells (w = 1 - r, r < 1; oercel.c:970-981) plus the
// harmonic bonds to prev/next (oercel.c:1272-1308).  Every pair is evaluated
// by both of its beads with exactly negated operands and summed in fixed point,
// so F_ij = -F_ji and sum F = 0 hold exactly and the result does not depend on
// the order of the loops.  The candidates of a thread are first screened
// (r < 1) into a per-thread list in shared memory, then the list is evaluated,
// so the expensive part (noise + force) runs without warp divergence on the
// cutoff test.  NEXTKEY: also the cell of x + dt vh + dt^2 F and its count,
// i.e. the first half of the next step's sort.
template <bool PAIR, bool BOND, bool NEXTKEY>
__global__ void __launch_bounds__(BEAD_TPB) k_forces(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                     const Chunk *__restrict__ ch) {
    pdl_begin();
    __shared__ float a_sh[DPD_MAXT * DPD_MAXT];
    __shared__ int hl[PAIR ? MAXHIT : 1][BEAD_TPB];
    const Chunk c = ch[blockIdx.x];
    const RepDev &R = reps[c.rep];
    if (threadIdx.x < DPD_MAXT * DPD_MAXT) a_sh[threadIdx.x] = a_at(R, threadIdx.x, *b.step);
    __syncthreads();
    const int d = c.begin + (int)threadIdx.x;
    const bool act = d < c.end;
    const float2 *__restrict__ pos = b.pos[cur];
    uint32_t key = 0;
    float mb = 0.0f;
    if (act) {
        long long ax = 0, ay = 0;
        const float2 pi = pos[d];
        const float L = R.L;
        if (PAIR) {
            PairCtx pc;
            pc.pos = pos;
            pc.vt = b.vt[cur];
            pc.tg = b.tg[cur];
            pc.pi = pi;
            pc.vi = pc.vt[d];
            const uint32_t tgi = pc.tg[d];
            pc.gi = tgi & GID_MASK;
            pc.arow = a_sh + (tgi >> TYPE_SHIFT) * DPD_MAXT;
            pc.nk = make_noise_key(R, *b.step);
            pc.L = L;
            pc.h = R.halfL;
            pc.gam = R.gamma;
            pc.sdt = sdt_at(R, *b.step);
            const int ncx = R.ncx, ncy = R.ncy;
            const int32_t *__restrict__ cs = b.cstart + R.c0;
            int cx, cy;
            cell_xy(R, pi.x, pi.y, cx, cy);
            int nh = 0;
#pragma unroll 1
            for (int ox = -1; ox <= 1; ox++) {
                int nx = cx + ox;
                float sx = 0.0f;
                if (nx < 0) {
                    nx += ncx;
                    sx = L;
                } else if (nx >= ncx) {
                    nx -= ncx;
                    sx = -L;
                }
                const int col = nx * ncy;
                // rows cy-1 .. cy+1 of this column: one or two contiguous slot ranges
                int s0, e0, s1 = 0, e1 = 0;
                float sy0 = 0.0f, sy1 = 0.0f;
                if (cy >= 1 && cy + 1 < ncy) {
                    s0 = cs[col + cy - 1];
                    e0 = cs[col + cy + 2];
                } else if (cy == 0) {
                    s0 = cs[col + ncy - 1];
                    e0 = cs[col + ncy];
                    sy0 = L;
                    s1 = cs[col];
                    e1 = cs[col + 2];
                } else {
                    s0 = cs[col + cy - 1];
                    e0 = cs[col + ncy];
                    s1 = cs[col];
                    e1 = cs[col + 1];
                    sy1 = -L;
                }
#pragma unroll 1
                for (int seg = 0; seg < 2; seg++) {
                    const int js = seg ? s1 : s0, je = seg ? e1 : e0;
                    const float sy = seg ? sy1 : sy0;
#pragma unroll 4
                    for (int j = js; j < je; j++) {
                        const float2 pj = pos[j];
                        const float dx = __fadd_rn(__fsub_rn(pi.x, pj.x), sx);
                        const float dy = __fadd_rn(__fsub_rn(pi.y, pj.y), sy);
                        const float r2 = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
                        if (r2 < 1.0f && r2 > 1e-24f && j != d) {
                            if (nh < MAXHIT) hl[nh][threadIdx.x] = j;
                            else pair_term(pc, j, ax, ay);  // crowded neighbourhood: evaluate at once
                            nh++;
                        }
                    }
                }
            }
            const int nl = min(nh, MAXHIT);
#pragma unroll 1
            for (int k = 0; k < nl; k++) pair_term(pc, hl[k][threadIdx.x], ax, ay);
            // the stirring body force belongs to the pair forces, as in the reference (oercel.c:1159-1165)
            if (R.stir_A != 0.0f) ax += stir_force(R, pi.y, pc.gi, b.stir[c.rep]);
        }
        if (BOND && R.arch != 0) {  // branched lipids: the template terms of k_mol_forces
            const int2 lk = b.link[cur][d];
            if (lk.x >= 0 || lk.y >= 0) {
                const int2 q = b.fmol[d];
                ax += q.x;
                ay += q.y;
            }
        } else if (BOND) {
            const int2 lk = b.link[cur][d];
            const float h = R.halfL, kb = R.kb, r0 = R.r0;
            float2 pjs[2];
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const int j = q ? lk.y : lk.x;
                pjs[q] = pi;
                if (j < 0) continue;
                const float2 pj = pos[j];
                pjs[q] = pj;
                const float dx = minimg(__fsub_rn(pj.x, pi.x), L, h), dy = minimg(__fsub_rn(pj.y, pi.y), L, h);
                const float r = __fsqrt_rn(__fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
                mb = fmaxf(mb, r);
                const float fb = __fdiv_rn(__fmul_rn(kb, __fsub_rn(r, r0)), r);
                ax += f2fix16(__fmul_rn(fb, dx));
                ay += f2fix16(__fmul_rn(fb, dy));
            }
            angle_terms(b, cur, R, pi, lk, pjs[0], pjs[1], ax, ay);
        }
        const float2 fs = make_float2(fix16_to_f(ax), fix16_to_f(ay));
        if (!(isfinite(fs.x) && isfinite(fs.y))) raise_flag(b.status, DPD_F_NONFINITE);
        b.f[cur][d] = fs;
        if (NEXTKEY) {
            const float2 v = b.vh[cur][d];
            int cx, cy;
            key = (uint32_t)(R.c0 + cell_xy(R, advance1(pi.x, v.x, fs.x, R.dt, R.dt2, L),
                                            advance1(pi.y, v.y, fs.y, R.dt, R.dt2, L), cx, cy));
        }
    }
    if (BOND) {
        // running max bond length of the replica (obs slot 4, float bits; r >= 0)
        const unsigned mbb = __reduce_max_sync(0xffffffffu, __float_as_uint(mb));
        if (lane_id() == 0 && mbb != 0u) atomicMax(b.obs + (size_t)c.rep * OBS_N + 4, (unsigned long long)mbb);
    }
    if (NEXTKEY) {
        count_key(b.count, key, act);
        if (act) b.key[d] = key;
    }
}

// vh = v - dt/2 f after the first force evaluation (oercel.c:2207-2211)
__global__ void __launch_bounds__(BEAD_TPB) k_halfkick(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                       const Chunk *__restrict__ ch) {
    const Chunk c = ch[blockIdx.x];
    const int d = c.begin + (int)threadIdx.x;
    if (d >= c.end) return;
    const float h = reps[c.rep].hdt;
    const float2 v = b.vh[cur][d], f = b.f[cur][d];
    b.vh[cur][d] = make_float2(__fmaf_rn(-h, f.x, v.x), __fmaf_rn(-h, f.y, v.y));
}

// the start of a step whose update keeps the slot order (the scan that does
// this on other steps is not launched): the step counter, and empty chemistry
// candidate lists
__global__ void k_step_begin(long long *__restrict__ step, DevStatus *__restrict__ status,
                             int32_t *__restrict__ resort, int nrep) {
    if (threadIdx.x == 0) {
        *step += 1;
        status->n_grow = 0u;
        status->n_bond = 0u;
    }
    for (int r = (int)threadIdx.x; r <= nrep; r += (int)blockDim.x) resort[r] = 0;
}

// the sorted copy (next buffer) of a sort before a catalyst check back into the
// current buffer, so that the buffer parity of the step does not depend on it
__global__ void __launch_bounds__(BEAD_TPB) k_copy_back(Bufs b, int cur, const Chunk *__restrict__ ch) {
    if (!b.resort[0]) return;
    const Chunk c = ch[blockIdx.x];
    const int d = c.begin + (int)threadIdx.x;
    if (d >= c.end) return;
    const int n = cur ^ 1;
    b.pos[cur][d] = b.pos[n][d];
    b.vh[cur][d] = b.vh[n][d];
    b.vt[cur][d] = b.vt[n][d];
    b.f[cur][d] = b.f[n][d];
    b.tg[cur][d] = b.tg[n][d];
    b.link[cur][d] = b.link[n][d];
}

// the Groot-Warren update in place, no sort (phase entry point dpd_integrate)
__global__ void __launch_bounds__(BEAD_TPB) k_integrate(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                        const Chunk *__restrict__ ch) {
    const Chunk c = ch[blockIdx.x];
    const int d = c.begin + (int)threadIdx.x;
    if (d >= c.end) return;
    const RepDev &R = reps[c.rep];
    const float2 p = b.pos[cur][d], vh = b.vh[cur][d], f = b.f[cur][d];
    const float2 q = make_float2(advance1(p.x, vh.x, f.x, R.dt, R.dt2, R.L), advance1(p.y, vh.y, f.y, R.dt, R.dt2, R.L));
    if (!(q.x >= 0.0f && q.x < R.L && q.y >= 0.0f && q.y < R.L)) raise_flag(b.status, DPD_F_OUTSIDE);
    b.pos[cur][d] = q;
    b.vt[cur][d] = make_float2(__fmaf_rn(R.cvt, f.x, vh.x), __fmaf_rn(R.cvt, f.y, vh.y));
    b.vh[cur][d] = make_float2(__fmaf_rn(R.dt, f.x, vh.x), __fmaf_rn(R.dt, f.y, vh.y));
}

// ---------------------------------------------------------------- observables

// per-bead sums (momentum, kinetic energy, type counts, chain heads) and the
// conservative virial over each unordered pair once; fixed-point integer sums
// make the result independent of the launch shape.  A grid-stride loop over
// the replica's chunks keeps each thread's sums in registers; a block reduction
// then leaves one atomic per quantity per block.
template <bool VIRIAL>
__global__ void __launch_bounds__(BEAD_TPB) k_observables(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                          const Chunk *__restrict__ ch, int rep_index,
                                                          unsigned long long *__restrict__ host_out,
                                                          int ring_slots) {
    __shared__ long long red[BEAD_TPB / 32][5 + DPD_MAXT];
    const RepDev &R = reps[rep_index];
    long long sx = 0, sy = 0, s2 = 0, vir = 0, heads = 0;
    int cnt[DPD_MAXT];
#pragma unroll
    for (int t = 0; t < DPD_MAXT; t++) cnt[t] = 0;
    // OBS_ITEMS chunks per round, their loads issued together (the chunk
    // descriptor, then the bead, are two dependent loads: more in flight)
    const int G = (int)gridDim.x;
    for (int k0 = (int)blockIdx.x; k0 < R.nch; k0 += OBS_ITEMS * G) {
        int d[OBS_ITEMS];
        bool act[OBS_ITEMS];
#pragma unroll
        for (int u = 0; u < OBS_ITEMS; u++) {
            const int k = k0 + u * G;
            act[u] = false;
            d[u] = 0;
            if (k < R.nch) {
                const Chunk c = ch[R.ch0 + k];
                d[u] = c.begin + (int)threadIdx.x;
                act[u] = d[u] < c.end;
            }
        }
        float2 v[OBS_ITEMS], f[OBS_ITEMS];
        uint32_t tgv[OBS_ITEMS];
        int2 lk[OBS_ITEMS];
#pragma unroll
        for (int u = 0; u < OBS_ITEMS; u++) {
            if (!act[u]) continue;
            v[u] = b.vh[cur][d[u]];
            f[u] = b.f[cur][d[u]];
            tgv[u] = b.tg[cur][d[u]];
            lk[u] = b.link[cur][d[u]];
        }
#pragma unroll
        for (int u = 0; u < OBS_ITEMS; u++) {
            if (!act[u]) continue;
            const double vx = (double)v[u].x + (double)R.hdt * (double)f[u].x;
            const double vy = (double)v[u].y + (double)R.hdt * (double)f[u].y;
            sx += __double2ll_rn(vx * OBS_FIX);
            sy += __double2ll_rn(vy * OBS_FIX);
            s2 += __double2ll_rn((vx * vx + vy * vy) * OBS_FIX);
            const int ty = (int)(tgv[u] >> TYPE_SHIFT);
#pragma unroll
            for (int t = 0; t < DPD_MAXT; t++) cnt[t] += ty == t;
            heads += (lk[u].x < 0 && lk[u].y >= 0) ? 1 : 0;
            // virial: pairs (d, j) with j > d inside the cutoff
            if (VIRIAL) {
                const int dd = d[u];
                const float2 *__restrict__ pos = b.pos[cur];
                const float2 pi = pos[dd];
                const int ncx = R.ncx, ncy = R.ncy;
                const int32_t *cs = b.cstart + R.c0;
                int cx, cy;
                cell_xy(R, pi.x, pi.y, cx, cy);
                double accv = 0.0;
                for (int ox = -1; ox <= 1; ox++)
                    for (int oy = -1; oy <= 1; oy++) {
                        const int nx = (cx + ox + ncx) % ncx, ny = (cy + oy + ncy) % ncy;
                        const int cc = nx * ncy + ny;
                        for (int j = cs[cc]; j < cs[cc + 1]; j++) {
                            if (j <= dd) continue;
                            const float2 pj = pos[j];
                            const double dx = (double)minimg(__fsub_rn(pi.x, pj.x), R.L, R.halfL);
                            const double dy = (double)minimg(__fsub_rn(pi.y, pj.y), R.L, R.halfL);
                            const double r2 = dx * dx + dy * dy;
                            if (!(r2 < 1.0 && r2 > 1e-24)) continue;
                            const double r = sqrt(r2);
                            accv += (double)a_at(R, ty * DPD_MAXT + (b.tg[cur][j] >> TYPE_SHIFT), *b.step) *
                                    (1.0 - r) * r;
                        }
                    }
                vir += __double2ll_rn(accv * OBS_FIX);
            }
        }
    }
    long long q[5 + DPD_MAXT] = {sx, sy, s2, vir, heads};
#pragma unroll
    for (int t = 0; t < DPD_MAXT; t++) q[5 + t] = cnt[t];
    const int lane = (int)lane_id(), w = (int)threadIdx.x >> 5;
#pragma unroll
    for (int e = 0; e < 5 + DPD_MAXT; e++) {
        const long long sum = warp_sum_ll(q[e]);
        if (lane == 0) red[w][e] = sum;
    }
    __syncthreads();
    if (threadIdx.x < 5 + DPD_MAXT) {
        long long sum = 0;
        for (int k = 0; k < BEAD_TPB / 32; k++) sum += red[k][threadIdx.x];
        // slots: 0, 1 momentum, 2 kinetic, 3 virial, 5 heads, 8 + t type counts (4 is the running max bond)
        const int slot = threadIdx.x < 4 ? (int)threadIdx.x : threadIdx.x == 4 ? 5 : 8 + (int)threadIdx.x - 5;
        if (sum != 0) atomicAdd(b.obs + (size_t)rep_index * OBS_N + slot, (unsigned long long)sum);
    }
    // the last block to finish hands the row over (to obs_out and, when given,
    // straight into the caller's pinned host buffer) and clears the sums for the
    // next row
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(b.obs_done + rep_index, 1u) == gridDim.x - 1;
    __syncthreads();
    if (last) {
        __threadfence();
        // a ring of rows in host memory: the slot of this step, its word 6 the step
        unsigned long long *out = host_out;
        const long long step = *b.step;
        if (out && ring_slots > 0) out += (size_t)(step % ring_slots) * OBS_N;
        if (threadIdx.x < OBS_N) {
            const unsigned long long v = atomicExch(b.obs + (size_t)rep_index * OBS_N + threadIdx.x, 0ull);
            b.obs_out[(size_t)rep_index * OBS_N + threadIdx.x] = v;
            if (out) out[threadIdx.x] = (ring_slots > 0 && threadIdx.x == 6) ? (unsigned long long)step : v;
        }
        if (threadIdx.x == 0) b.obs_done[rep_index] = 0u;
    }
}

// distances between types ta and tb (ta < 0: all beads) within rmax (<= 3
// cells), each unordered pair once, binned as the reference's `snapcheck.py
// rdf` bins them (np.histogram over [0, rmax] of pairs with d <= rmax,
// cel/engine/tests/snapcheck.py:86-107): d in FP64 from the FP32 positions with
// the minimum image, the bin from d * nbin / rmax corrected against the edges
// k * (rmax / nbin), the last bin closed on the right
__global__ void __launch_bounds__(BEAD_TPB) k_pair_hist(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                        const Chunk *__restrict__ ch, int rep_index, int ta, int tb,
                                                        double rmax, int nbin) {
    const Chunk c = ch[blockIdx.x];
    if (c.rep != rep_index) return;
    const RepDev &R = reps[c.rep];
    const int d = c.begin + (int)threadIdx.x;
    if (d >= c.end) return;
    const int ti = (int)(b.tg[cur][d] >> TYPE_SHIFT);
    if (ta >= 0 && ti != ta && ti != tb) return;
    const float2 *__restrict__ pos = b.pos[cur];
    const float2 pi = pos[d];
    const int ncx = R.ncx, ncy = R.ncy;
    const int rc = (int)ceil(rmax * R.icsx);
    const int rx = min(rc, (ncx - 1) / 2), ry = min(rc, (ncy - 1) / 2);
    const int32_t *cs = b.cstart + R.c0;
    const double L = (double)R.L, norm = (double)nbin / rmax, step = rmax / (double)nbin;
    int cx, cy;
    cell_xy(R, pi.x, pi.y, cx, cy);
    for (int ox = -rx; ox <= rx; ox++)
        for (int oy = -ry; oy <= ry; oy++) {
            const int nx = (cx + ox + ncx) % ncx, ny = (cy + oy + ncy) % ncy;
            const int cc = nx * ncy + ny;
            for (int j = cs[cc]; j < cs[cc + 1]; j++) {
                if (j <= d) continue;
                const int tj = (int)(b.tg[cur][j] >> TYPE_SHIFT);
                if (ta >= 0 && !((ti == ta && tj == tb) || (ti == tb && tj == ta))) continue;
                const float2 pj = pos[j];
                double dx = (double)pi.x - (double)pj.x, dy = (double)pi.y - (double)pj.y;
                dx -= L * rint(dx / L);
                dy -= L * rint(dy / L);
                const double r = hypot(dx, dy);
                if (!(r <= rmax)) continue;
                int bin = (int)(r * norm);
                if (bin >= nbin) bin = nbin - 1;
                if (r < bin * step) bin--;
                else if (bin + 1 < nbin && r >= (bin + 1) * step) bin++;
                if (bin >= 0 && bin < nbin) atomicAdd(b.hist + bin, 1ull);
            }
        }
}

// ---------------------------------------------------------------- state in/out

// a bead handed in: a finite position is wrapped into [0, L) (values inside are
// kept as they are; a float32 snapshot coordinate may round to exactly L);
// a non-finite position, a type >= DPD_MAXT, a gid >= n or a link outside
// [-1, n) is stored sanitised and flagged (DPD_F_INPUT), so nothing out of range
// ever reaches the step's kernels
__global__ void k_pack(Bufs b, int cur, int b0, int n, float L, const float *x, const float *y, const float *vx,
                       const float *vy, const uint8_t *type, const uint32_t *gid, const int32_t *prev,
                       const int32_t *next) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int d = b0 + k;
    float px = x[k], py = y[k];
    uint32_t t = type[k], g = gid ? gid[k] : (uint32_t)k;
    int p = prev ? prev[k] : -1, q = next ? next[k] : -1;
    bool bad = false;
    if (!(isfinite(px) && isfinite(py))) {
        px = py = 0.0f;
        bad = true;
    }
    if (!(px >= 0.0f && px < L)) {
        px = fmodf(px, L);
        px = px < 0.0f ? px + L : px;
        px = px >= L ? 0.0f : px;
    }
    if (!(py >= 0.0f && py < L)) {
        py = fmodf(py, L);
        py = py < 0.0f ? py + L : py;
        py = py >= L ? 0.0f : py;
    }
    if (t >= (uint32_t)DPD_MAXT) {
        t = 0;
        bad = true;
    }
    if (g >= (uint32_t)n) {
        g = (uint32_t)k;
        bad = true;
    }
    if (p < -1 || p >= n || q < -1 || q >= n) {
        p = q = -1;
        bad = true;
    }
    if (bad) raise_flag(b.status, DPD_F_INPUT);
    b.pos[cur][d] = make_float2(px, py);
    b.vh[cur][d] = make_float2(vx[k], vy[k]);
    b.vt[cur][d] = make_float2(vx[k], vy[k]);
    b.f[cur][d] = make_float2(0.0f, 0.0f);
    b.tg[cur][d] = (t << TYPE_SHIFT) | (g & GID_MASK);
    b.link[cur][d] = make_int2(p >= 0 ? b0 + p : -1, q >= 0 ? b0 + q : -1);
}

__global__ void k_unpack(Bufs b, int cur, int b0, int n, float *x, float *y, float *vhx, float *vhy, float *vtx,
                         float *vty, float *fx, float *fy, uint8_t *type, uint32_t *gid, int32_t *prev,
                         int32_t *next) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int d = b0 + k;
    const float2 p = b.pos[cur][d], vh = b.vh[cur][d], vt = b.vt[cur][d], f = b.f[cur][d];
    if (x) x[k] = p.x;
    if (y) y[k] = p.y;
    if (vhx) vhx[k] = vh.x;
    if (vhy) vhy[k] = vh.y;
    if (vtx) vtx[k] = vt.x;
    if (vty) vty[k] = vt.y;
    if (fx) fx[k] = f.x;
    if (fy) fy[k] = f.y;
    const uint32_t tg = b.tg[cur][d];
    if (type) type[k] = (uint8_t)(tg >> TYPE_SHIFT);
    if (gid) gid[k] = tg & GID_MASK;
    const int2 lk = b.link[cur][d];
    if (prev) prev[k] = lk.x >= 0 ? lk.x - b0 : -1;
    if (next) next[k] = lk.y >= 0 ? lk.y - b0 : -1;
}

__global__ void k_set_dynamics(Bufs b, int cur, int b0, int n, const float *vhx, const float *vhy, const float *fx,
                               const float *fy, const float *vtx, const float *vty) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int d = b0 + k;
    float2 v = b.vh[cur][d], f = b.f[cur][d], t = b.vt[cur][d];
    if (vhx) v.x = vhx[k];
    if (vhy) v.y = vhy[k];
    if (fx) f.x = fx[k];
    if (fy) f.y = fy[k];
    if (vtx) t.x = vtx[k];
    if (vty) t.y = vty[k];
    b.vh[cur][d] = v;
    b.f[cur][d] = f;
    b.vt[cur][d] = t;
}

// ---------------------------------------------------------------- launchers

void launch_keys(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, bool integrate,
                 cudaStream_t s) {
    if (integrate) k_keys<true, false><<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch);
    else k_keys<false, false><<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch);
}

static void scan_part(const Bufs &b, int64_t C, bool step_inc, int part, const int32_t *gate, cudaStream_t s) {
    const int nb = (int)((C + SCAN_PER_BLOCK - 1) / SCAN_PER_BLOCK);
    if (part == 1)
        launch_pdl(k_scan1<true>, nb, SCAN_TPB, 0, s, b.count, b.cstart, b.bsum, (long long)C, b.step,
                   step_inc ? 1 : 0, b.status, gate);
    else launch_pdl(k_scan2, nb, SCAN_TPB, 0, s, b.cstart, b.fill, b.bsum, (long long)C, nb, gate);
}

void launch_scan_part(const Bufs &b, int64_t C, bool step_inc, int part, cudaStream_t s) {
    scan_part(b, C, step_inc, part, nullptr, s);
}

void launch_scan_lb(const Bufs &b, int64_t C, bool step_inc, cudaStream_t s) {
    const int nb = (int)((C + SCAN_PER_BLOCK - 1) / SCAN_PER_BLOCK);
    launch_pdl(k_scan_lb, nb, SCAN_TPB, 0, s, b.count, b.cstart, b.fill, b.scan_state, b.scan_ticket, (long long)C, nb,
               b.step, step_inc ? 1 : 0, b.status);
}

void launch_scan(const Bufs &b, int64_t C, bool step_inc, cudaStream_t s) {
    launch_scan_part(b, C, step_inc, 1, s);
    launch_scan_part(b, C, step_inc, 2, s);
}

void launch_place(const Bufs &b, const Chunk *bch, int nbch, cudaStream_t s) {
    launch_pdl(k_place<false>, (nbch + PLACE_ITEMS - 1) / PLACE_ITEMS, BEAD_TPB, 0, s, b, bch, nbch,
               (const int32_t *)nullptr, 0);
}

void launch_cellfix(const Bufs &b, const Chunk *cch, int ncch, cudaStream_t s) {
    launch_pdl(k_cellfix<false>, ncch, CELL_TPB, 0, s, b, cch, (const int32_t *)nullptr, 0, 0ll);
}

bool sort_pfx_fits(int64_t C) { return (C + SCAN_PER_BLOCK - 1) / SCAN_PER_BLOCK <= PFX_MAX; }

void launch_sort_pfx(const Bufs &b, int64_t C, bool step_inc, const Chunk *bch, int nbch, const Chunk *cch, int ncch,
                     int part, cudaStream_t s) {
    const int nb = (int)((C + SCAN_PER_BLOCK - 1) / SCAN_PER_BLOCK);
    const int32_t *no = nullptr;
    if (part < 0 || part == 0)
        launch_pdl(k_scan1<false>, nb, SCAN_TPB, 0, s, b.count, (int32_t *)b.fill, b.bsum, (long long)C, b.step,
                   step_inc ? 1 : 0, b.status, no);
    if (part < 0 || part == 1)
        launch_pdl(k_place<true>, (nbch + PLACE_ITEMS - 1) / PLACE_ITEMS, BEAD_TPB, 0, s, b, bch, nbch, no, nb);
    if (part < 0 || part == 2) launch_pdl(k_cellfix<true>, ncch, CELL_TPB, 0, s, b, cch, no, nb, (long long)C);
}

void launch_permute(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, PermuteMode mode,
                    cudaStream_t s) {
    const int g4 = (nbch + PERM_ITEMS - 1) / PERM_ITEMS;
    const int32_t *no = nullptr;
    if (mode == PERM_STEP) launch_pdl(k_permute<PERM_STEP, PERM_ITEMS>, g4, BEAD_TPB, 0, s, b, cur, rep, bch, nbch, no);
    else if (mode == PERM_KEEP)
        launch_pdl(k_permute<PERM_KEEP, PERM_ITEMS>, g4, BEAD_TPB, 0, s, b, cur, rep, bch, nbch, no);
    else if (mode == PERM_PRIME) k_permute<PERM_PRIME, 1><<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch, nbch, no);
    else k_permute<PERM_SORT, 1><<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch, nbch, no);
}

// The reference sorts again before a catalyst check when a bead moved 0.5 or
// more in the step (oercel.c:2339-2344).  The kernels below run as no-ops
// unless k_permute<PERM_KEEP> flagged a replica; then the flagged replicas are
// sorted by their new positions (the others keep their order), and the sorted
// state is copied back so the host's buffer parity stays the same.
void launch_resort(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, const Chunk *cch, int ncch,
                   int64_t C, cudaStream_t s) {
    const int32_t *gate = b.resort;
    cudaMemsetAsync(b.count, 0, (size_t)(C + 4) * sizeof(uint32_t), s);
    k_keys<false, true><<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch);
    scan_part(b, C, false, 1, gate, s);
    scan_part(b, C, false, 2, gate, s);
    launch_pdl(k_place<false>, (nbch + PLACE_ITEMS - 1) / PLACE_ITEMS, BEAD_TPB, 0, s, b, bch, nbch, gate, 0);
    launch_pdl(k_cellfix<false>, ncch, CELL_TPB, 0, s, b, cch, gate, 0, 0ll);
    k_permute<PERM_SORT, 1><<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch, nbch, gate);
    k_copy_back<<<nbch, BEAD_TPB, 0, s>>>(b, cur, bch);
}

void launch_forces(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, bool pair, bool bond,
                   bool next_keys, cudaStream_t s) {
    if (pair && bond && next_keys) launch_pdl(k_forces<true, true, true>, nbch, BEAD_TPB, 0, s, b, cur, rep, bch);
    else if (pair && bond) k_forces<true, true, false><<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch);
    else if (pair) k_forces<true, false, false><<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch);
    else k_forces<false, true, false><<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch);
}

void launch_halfkick(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, cudaStream_t s) {
    k_halfkick<<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch);
}

// The event log read without a wait: the events recorded since the last read
// are copied into the caller's host buffer (at most cap of them, the device can
// write it), then k_events_done writes how many were recorded (cap exceeded
// too) and clears the log.  Both run on the stream, after the steps before them.
__global__ void k_events_out(const EventDev *__restrict__ ev, const DevStatus *__restrict__ st, int evcap,
                             EventDev *__restrict__ out, int cap) {
    const int m = min((int)min(st->nevents, (unsigned)evcap), cap);
    for (int i = (int)(blockIdx.x * blockDim.x + threadIdx.x); i < m; i += (int)(gridDim.x * blockDim.x))
        out[i] = ev[i];
}

__global__ void k_events_done(DevStatus *__restrict__ st, int *__restrict__ n_out) {
    *n_out = (int)st->nevents;
    st->nevents = 0u;
}

void launch_events_out(const Bufs &b, EventDev *out, int cap, int *n_out, cudaStream_t s) {
    k_events_out<<<16, 256, 0, s>>>(b.events, b.status, b.evcap, out, cap);
    k_events_done<<<1, 1, 0, s>>>(b.status, n_out);
}

void launch_step_begin(const Bufs &b, int nrep, cudaStream_t s) {
    k_step_begin<<<1, 128, 0, s>>>(b.step, b.status, b.resort, nrep);
}

void launch_integrate(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, cudaStream_t s) {
    k_integrate<<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch);
}

void launch_observables(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, int rep_index,
                        bool virial, unsigned long long *host_out, int ring_slots, cudaStream_t s) {
    const int grid = std::min(nbch, 148 * 8);  // grid-stride over the replica's chunks
    if (virial) k_observables<true><<<grid, BEAD_TPB, 0, s>>>(b, cur, rep, bch, rep_index, host_out, ring_slots);
    else k_observables<false><<<grid, BEAD_TPB, 0, s>>>(b, cur, rep, bch, rep_index, host_out, ring_slots);
}

void launch_pair_hist(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, int rep_index, int ta,
                      int tb, double rmax, int nbin, cudaStream_t s) {
    k_pair_hist<<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch, rep_index, ta, tb, rmax, nbin);
}

void launch_pack(const Bufs &b, int cur, int b0, int n, float L, const float *x, const float *y, const float *vx,
                 const float *vy, const uint8_t *type, const uint32_t *gid, const int32_t *prev,
                 const int32_t *next, cudaStream_t s) {
    k_pack<<<(n + 255) / 256, 256, 0, s>>>(b, cur, b0, n, L, x, y, vx, vy, type, gid, prev, next);
}

void launch_unpack(const Bufs &b, int cur, int b0, int n, float *x, float *y, float *vhx, float *vhy, float *vtx,
                   float *vty, float *fx, float *fy, uint8_t *type, uint32_t *gid, int32_t *prev, int32_t *next,
                   cudaStream_t s) {
    k_unpack<<<(n + 255) / 256, 256, 0, s>>>(b, cur, b0, n, x, y, vhx, vhy, vtx, vty, fx, fy, type, gid, prev, next);
}

void launch_set_dynamics(const Bufs &b, int cur, int b0, int n, const float *vhx, const float *vhy,
                         const float *fx, const float *fy, const float *vtx, const float *vty, cudaStream_t s) {
    k_set_dynamics<<<(n + 255) / 256, 256, 0, s>>>(b, cur, b0, n, vhx, vhy, fx, fy, vtx, vty);
}
