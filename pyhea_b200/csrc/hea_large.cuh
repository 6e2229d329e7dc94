// hea_large.cuh -- the search for structures whose occupancy does not fit in
// shared memory (up to millions of sites).
//
// Same contract as hea_search.cuh (Philox streams, counts, fitness order,
// ties), so results are bit-identical to the shared-memory path; only where
// the occupancy lives and how many SMs work on one solution change:
//   * the occupancy row stays in HBM as species bytes; the local search does
//     not read or write it: its draws take the species from the site
//     histograms' species words (hist[s].w = 5*species), which the accepts
//     keep current, and at its end each CTA writes its share of the row back
//     from those words;
//   * one thread-block cluster per solution: the round's tasks are split over
//     the cluster's CTAs; each CTA reduces its warps' records, publishes its
//     best in shared memory, and after one cluster barrier every warp reads the
//     CL records through distributed shared memory and applies the same winner;
//   * generation and recount are grid-wide over sites (many CTAs per solution);
//     the recount also writes the site histograms the search scores from
//     (hist, see score_delta), which rank 0 of the cluster updates after every
//     accepted swap, followed by a cluster barrier that only rank 0 arrives at
//     with release semantics (the other CTAs have nothing to publish).
#pragma once
#include <cooperative_groups.h>

#include "hea_search.cuh"

namespace hea {

namespace cg = cooperative_groups;

// Random occupancy of population positions [0, count) of `generation` into
// slot rows order[pos], as species bytes.  grid = (chunks, count).
template <int T>
__global__ void __launch_bounds__(256) large_generate_kernel(const SearchConst c, uint8_t *occ, const int32_t *order,
                                                             uint32_t generation)
{
    const uint32_t pos = blockIdx.y;
    uint8_t *row = occ + (size_t)order[pos] * c.occ_stride;
    uint32_t rk[kFeistelRounds];
    const u32x4 w0 = philox4x32_10(u32x4{pos, generation, 0u, kInitStream}, c.key0, c.key1);
    const u32x4 w1 = philox4x32_10(u32x4{pos, generation, 1u, kInitStream}, c.key0, c.key1);
    rk[0] = w0.x; rk[1] = w0.y; rk[2] = w0.z; rk[3] = w0.w; rk[4] = w1.x; rk[5] = w1.y;
    const int n = c.num_sites;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        uint32_t y = feistel((uint32_t)s, c.feistel_h, rk);
        while (y >= (uint32_t)n) y = feistel(y, c.feistel_h, rk);
        int t = 0;
#pragma unroll
        for (int i = 1; i < T; ++i) t += (int)(y >= (uint32_t)c.prefix[i]);
        row[s] = (uint8_t)t;
    }
}

// Pair counts of slot rows order[pos] (species bytes), accumulated into
// cnt[order[pos]] (zeroed by the caller), and, with `hist`, the site
// histograms of those rows (hist + slot * N; see block_recount).  grid =
// (chunks, count); each CTA counts a range of sites into shared bins and adds
// them once.
template <int T, int S>
__global__ void __launch_bounds__(256) large_recount_kernel(const SearchConst c, const int4 *__restrict__ nbor,
                                                            const uint8_t *occ, const int32_t *order, int32_t *cnt,
                                                            uint4 *hist)
{
    __shared__ int32_t bins[S * T * T];
    const int slot = order[blockIdx.y];
    const uint8_t *row = occ + (size_t)slot * c.occ_stride;
    for (int x = threadIdx.x; x < S * T * T; x += blockDim.x) bins[x] = 0;
    __syncthreads();
    const int n = c.num_sites;
    uint4 *hs = hist ? hist + (size_t)slot * n : nullptr;
    // one site with its shell histograms h (5-bit fields)
    const auto site = [&](int s, const uint32_t (&h)[S]) {
        const int a = row[s];
        uint32_t hk[3] = {0u, 0u, 0u};
#pragma unroll
        for (int k = 0; k < S; ++k) {
#pragma unroll
            for (int t = 0; t < T; ++t) {
                const int v = (int)((h[k] >> (5 * t)) & 31u);
                if (v) atomicAdd(&bins[(k * T + a) * T + t], v);
            }
            hk[k] = h[k] - (uint32_t)c.pad[k];  // sentinel entries counted as species 0
        }
        if (hs) hs[s] = make_uint4(hk[0], hk[1], hk[2], (uint32_t)(5 * a));  // species word: 5*species
    };
    const int first = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    if (c.lat.L) {  // implicit neighbours (no sentinel padding: pad[k] == 0)
        lattice_sites<S, uint32_t>(c.lat, first, stride, [row](int n) { return 1u << (5 * row[n]); }, site);
    } else {
        for (int s = first; s < n; s += stride) {
            uint32_t h[S];
#pragma unroll
            for (int k = 0; k < S; ++k) {
                h[k] = 0;
                const int4 *seg = nbor + (size_t)s * c.row4 + c.off4[k];
                for (int ch = 0; ch < c.chunks[k]; ++ch) {
                    const int4 x = __ldg(seg + ch);
                    h[k] += (1u << (5 * row[x.x])) + (1u << (5 * row[x.y])) + (1u << (5 * row[x.z])) +
                            (1u << (5 * row[x.w]));
                }
            }
            site(s, h);
        }
    }
    __syncthreads();
    int32_t *g = cnt + (size_t)slot * S * T * T;
    for (int x = threadIdx.x; x < S * T * T; x += blockDim.x) {
        int v = bins[x];
        if (blockIdx.x == 0 && x % T == 0) {  // sentinel entries land in field 0: pad_k per site of species i
            const int k = x / (T * T), i = (x / T) % T;
            v -= c.pad[k] * (c.prefix[i + 1] - c.prefix[i]);
        }
        if (v) atomicAdd(&g[x], v);
    }
}

// f2 of slots order[0, count) from their counts.
template <int T, int S>
__global__ void large_fitness_kernel(const SearchConst c, const int32_t *order, int count, const int32_t *cnt,
                                     double *f2)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) return;
    const int slot = order[p];
    f2[slot] = fitness_of_counts<T, S>(c, cnt + (size_t)slot * S * T * T);
}

// The local search with the occupancy in HBM, one cluster per solution.
// Shared memory: search_smem_tail(T, S, nwarps) + 2 * sizeof(SwapRecord):
// delta table, the warps' records [2][nwarps], two count buffers, and this
// CTA's best record [2] (read by the cluster).  Every CTA keeps its own copy of
// the table and counts and applies each accepted swap to them itself.
template <int T, class L>
__global__ void __launch_bounds__(512, 2) mc_large_kernel(const SearchConst c, const McArgs g)
{
    constexpr int S = L::S, NC = S * T * T, NCP = mc_ncount_pad(NC);
    extern __shared__ __align__(16) uint8_t smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank(), csize = (int)cluster.num_blocks();
    const int sol = blockIdx.x / csize;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    double2 *tab = reinterpret_cast<double2 *>(smem);
    SwapRecord *rec = reinterpret_cast<SwapRecord *>(tab + delta_entries(T, S));  // [2][nwarps]
    int32_t *cnt2 = reinterpret_cast<int32_t *>(rec + 2 * nwarps);                // [2][NCP]
    SwapRecord *cta_rec = reinterpret_cast<SwapRecord *>(cnt2 + 2 * NCP);         // [2]: this CTA's best

    const int slot = g.order[sol];
    const uint32_t stream = (g.mc_call << 16) | (uint32_t)sol;
    uint8_t *row = g.occ + (size_t)slot * c.occ_stride;
    uint4 *hist = g.hist + (size_t)slot * c.num_sites;
    int32_t *gcnt = g.cnt + (size_t)slot * NC;
    const int n = c.num_sites;
    // this CTA's share of the row and of the tasks
    const int part = (n + csize - 1) / csize, lo = rank * part, hi = min(n, lo + part);
    const int qpart = (g.tasks + csize - 1) / csize, qlo = rank * qpart, qhi = min(g.tasks, qlo + qpart);

    for (int x = tid; x < NC; x += blockDim.x) cnt2[x] = gcnt[x];
    __syncthreads();
    search_setup<T, S>(c, cnt2, tab);
    cluster.sync();

    double cur = g.f2[slot];
    int miss = 0, buf = 0;
    int64_t round = 0, accepts = 0, evals = 0;
    while (miss < g.depth && round < g.max_rounds) {
        SwapRecord *rr = rec + (round & 1) * nwarps;
        SwapRecord &mine = rr[warp];
        if (lane == 0) {
            mine.key = kNoSwap;
            mine.task = 0x7FFFFFFF;
        }
        __syncwarp();
        for (int q0 = qlo + warp * 32; q0 < qhi; q0 += blockDim.x) {
            const int q = q0 + lane;
            uint32_t s1 = 0, s2 = 0;
            uint4 hp = make_uint4(0u, 0u, 0u, 0u), hq = hp;
            // the species come from the histograms' species words: one L2 round trip per attempt
            const bool ok = q < qhi && draw_pair_hist(c, stream, (uint32_t)round, (uint32_t)q, hist, s1, s2, hp, hq);
            __syncwarp();
            uint64_t key = kNoSwap;
            uint32_t h1[S], h2[S];
            int a = 0, b = 0;
            if (ok) {
                ++evals;
                a = (int)hp.w / 5;
                b = (int)hq.w / 5;
                key = delta_key(score_delta<T, L>(c, g.nbor, g.nbmask, tab, hp, hq, s1, s2, a, b, h1, h2));
            }
            uint64_t wk = key;
            int wq = key != kNoSwap ? q : 0x7FFFFFFF;
            warp_argmin(wk, wq);
            if (key != kNoSwap && wq == q && better(wk, wq, mine.key, mine.task)) {
                SwapRecord r;
                r.key = wk;
                r.task = wq;
                r.s1 = s1;
                r.s2 = s2;
                r.ab = a | (b << 8);
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    r.h1[k] = k < S ? h1[k < S ? k : 0] : 0;
                    r.h2[k] = k < S ? h2[k < S ? k : 0] : 0;
                }
                r.stop = 0;
                r.pad_ = 0;
                mine = r;
            }
            __syncwarp();
        }
        __syncthreads();
        // this CTA's best record, published for the cluster
        if (warp == 0) {
            uint64_t xk = lane < nwarps ? rr[lane].key : kNoSwap;
            int xq = lane < nwarps ? rr[lane].task : 0x7FFFFFFF;
            const uint64_t own_k = xk;
            const int own_q = xq;
            warp_argmin(xk, xq);
            const int xw = __ffs(__ballot_sync(0xFFFFFFFFu, own_k == xk && own_q == xq)) - 1;
            if (lane == 0) cta_rec[round & 1] = rr[xw];
        }
        cluster.sync();
        // every warp reduces the cluster's records
        uint64_t xk = kNoSwap;
        int xq = 0x7FFFFFFF;
        if (lane < csize) {
            const SwapRecord *remote = cluster.map_shared_rank(&cta_rec[round & 1], lane);
            xk = remote->key;
            xq = remote->task;
        }
        const uint64_t own_k = xk;
        const int own_q = xq;
        warp_argmin(xk, xq);
        if (xk != kNoSwap) {
            const int xr = __ffs(__ballot_sync(0xFFFFFFFFu, own_k == xk && own_q == xq)) - 1;
            const SwapRecord w = *cluster.map_shared_rank(&cta_rec[round & 1], xr);
            const int a = w.ab & 0xFF, b = (w.ab >> 8) & 0xFF;
            const int32_t *cold = cnt2 + buf * NCP;
            int32_t *cnew = cnt2 + (buf ^ 1) * NCP;
            const auto after = [cold, &w, a, b](int k, int i, int j) {
                return cold[(k * T + i) * T + j] + count_change<T>(w, a, b, k, i, j);
            };
            const int me = block_rotation(32 * accept_linear_warps<T, S>());
            for (int x = me; x < NC; x += blockDim.x) cnew[x] = after(x / (T * T), (x / T) % T, x % T);
            delta_linear<T, S>(c, tab, after);
            if (rank == 0)
                update_hist<L, true>(c, g.nbor, hist, w.s1, w.s2, a, b,
                                     block_rotation(32 * (accept_linear_warps<T, S>() + (NC + 31) / 32)));
            // the cluster's next proposals read the histograms and species words rank 0 updated: rank 0
            // arrives with release semantics, the others (whose accept work stays in their own shared
            // memory) relaxed, every thread waits with acquire semantics.  Measured: 4 % per round.
            if (rank == 0)
                asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
            else
                asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
            asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
            buf ^= 1;
            cur = __dadd_rn(cur, key_delta(xk));
            if (g.trace && rank == 0 && warp == 0 && accepts < g.trace_cap) {
                if (lane == 0) {
                    AcceptRecord r;
                    r.round = (uint32_t)round;
                    r.task = (uint32_t)xq;
                    r.s1 = w.s1;
                    r.s2 = w.s2;
                    r.f2 = cur;
                    g.trace[(size_t)sol * g.trace_cap + accepts] = r;
                }
                if (g.trace_counts) {
                    int32_t *dst = g.trace_counts + ((size_t)sol * g.trace_cap + accepts) * NC;
                    for (int x = lane; x < NC; x += 32) dst[x] = cnew[x];
                }
            }
            miss = 0;
            ++accepts;
        } else {
            ++miss;
        }
        ++round;
    }
    cluster.sync();  // rank 0's last species words are visible
    for (int s = lo + tid; s < hi; s += blockDim.x) row[s] = (uint8_t)(__ldcg(&hist[s].w) / 5u);
    if (rank == 0)
        for (int x = tid; x < NC; x += blockDim.x) gcnt[x] = cnt2[buf * NCP + x];
    unsigned long long ev = (unsigned long long)evals;
#pragma unroll
    for (int o = 16; o; o >>= 1) ev += __shfl_xor_sync(0xFFFFFFFFu, ev, o);
    if (lane == 0 && ev) atomicAdd(&g.stats[1], ev);
    if (rank == 0 && tid == 0) {
        g.f2[slot] = fitness_of_counts<T, S>(c, cnt2 + buf * NCP);
        atomicAdd(&g.stats[0], (unsigned long long)round);
        atomicAdd(&g.stats[2], (unsigned long long)accepts);
        if (g.trace_len) g.trace_len[sol] = accepts;
        if (g.rounds_out) g.rounds_out[sol] = round;
    }
    cluster.sync();  // keep every CTA's shared memory alive until all remote reads are done
}

}  // namespace hea
