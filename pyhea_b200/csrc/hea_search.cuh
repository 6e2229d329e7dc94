// hea_search.cuh -- the swap-search kernels (sm_100a), templated on the number
// of species T and of shells S.
//
// Layout in HBM (one structure):
//   nbor   int32 [N][row] with every shell segment padded to a multiple of 4
//          entries by the sentinel site N, so each segment is read as int4
//   occ    uint8 [slots][occ_stride]   species per site, one row per slot
//   cnt    int32 [slots][S][T][T]      pair counts that travel with their slot
//   f2     double [slots]              squared weighted SRO error
//   order  int32 [2P]                  slot ids: current population, then the new one
// In shared memory a slot's occupancy is held as 5*species (the shift of its
// 5-bit histogram field), plus the sentinel byte 0 at index N.
#pragma once
#include <cstdint>

#include "hea_device.cuh"

namespace hea {

struct SearchConst {
    double E[kMaxShells * kMaxTypes * kMaxTypes];  // 1 - target, [S][T][T] compact
    double R[kMaxShells * kMaxTypes * kMaxTypes];  // N / (Z_k n_i n_j), [S][T][T] compact
    double w[kMaxShells];
    int32_t off4[kMaxShells];     // shell segment start in a row, int4 units
    int32_t chunks[kMaxShells];   // shell segment length, int4 units
    int32_t pad[kMaxShells];      // sentinel entries in the segment
    int32_t prefix[kMaxTypes + 1];  // species prefix sums
    int32_t num_sites, row4, occ_stride, num_types, num_shells, feistel_h;
    uint32_t reject_below, key0, key1;
};

struct AcceptRecord {
    uint32_t round, task, s1, s2;
    double f2;
};

struct McArgs {
    const int4 *nbor;
    uint8_t *occ;
    int32_t *cnt;
    double *f2;
    const int32_t *order;  // slots searched by this launch, one CTA each
    uint32_t mc_call;
    int32_t tasks, depth;
    int64_t max_rounds;
    unsigned long long *stats;  // [0] rounds, [1] evals, [2] accepts
    // optional trace (tests): per CTA up to trace_cap records and count snapshots
    AcceptRecord *trace;
    int32_t *trace_counts;
    int64_t *trace_len;
    int64_t trace_cap;
    int64_t *rounds_out;  // optional, per CTA
};

struct GenArgs {
    const int4 *nbor;
    uint8_t *occ;
    int32_t *cnt;
    double *f2;
    const int32_t *order;
    uint32_t generation;
    int32_t generate;  // 1: draw a new occupancy; 0: recount the stored one
};

// ---------------------------------------------------------------------------
// Fitness: f2 = sum_k w_k sum_i sum_j d^2, d = fma(-C', R, E), in k, i, j order.
// ---------------------------------------------------------------------------
template <int T, int S>
__device__ __forceinline__ double fitness_of_counts(const SearchConst &c, const int32_t *cnt)
{
    double f2 = 0.0;
#pragma unroll
    for (int k = 0; k < S; ++k) {
        double e = 0.0;
#pragma unroll
        for (int x = 0; x < T * T; ++x) {
            const int idx = k * T * T + x;
            const double d = __fma_rn(-(double)cnt[idx], c.R[idx], c.E[idx]);
            e = __fma_rn(d, d, e);
        }
        f2 = __fma_rn(c.w[k], e, f2);
    }
    return f2;
}

// Packed 5-bit species histogram of one padded shell segment of a row, and
// the number of entries equal to `other`.
template <bool COUNT_OTHER>
__device__ __forceinline__ uint32_t segment_hist(const int4 *__restrict__ seg, int chunks, const uint8_t *occ5,
                                                 uint32_t other, int &m)
{
    uint32_t h = 0;
    for (int ch = 0; ch < chunks; ++ch) {
        const int4 x = __ldg(seg + ch);
        h += (1u << occ5[x.x]) + (1u << occ5[x.y]) + (1u << occ5[x.z]) + (1u << occ5[x.w]);
        if (COUNT_OTHER)
            m += ((uint32_t)x.x == other) + ((uint32_t)x.y == other) + ((uint32_t)x.z == other) +
                 ((uint32_t)x.w == other);
    }
    return h;
}

// Row/column delta vector u of shell k for swapping species a (at s1) and b
// (at s2): u_t = n2_t - n1_t + m([t==b] - [t==a]); the count change is
// dC_ij = sa_i u_j + sa_j u_i with sa_i = [i==a] - [i==b].
template <int T>
__device__ __forceinline__ void delta_vector(uint32_t h1, uint32_t h2, int m, int a, int b, int (&u)[T])
{
#pragma unroll
    for (int t = 0; t < T; ++t) {
        u[t] = (int)((h2 >> (5 * t)) & 31u) - (int)((h1 >> (5 * t)) & 31u);
        u[t] += (t == b ? m : 0) - (t == a ? m : 0);
    }
}

// Score one proposal: f2 of the counts after swapping s1 (species a) and s2 (b).
template <int T, int S>
__device__ __forceinline__ double score_swap(const SearchConst &c, const int4 *__restrict__ nbor, const uint8_t *occ5,
                                             const int32_t *cnt, uint32_t s1, uint32_t s2, int a, int b,
                                             uint32_t (&h1)[S], uint32_t (&h2)[S], int (&m)[S])
{
    const int4 *r1 = nbor + (size_t)s1 * c.row4;
    const int4 *r2 = nbor + (size_t)s2 * c.row4;
    double f2 = 0.0;
#pragma unroll
    for (int k = 0; k < S; ++k) {
        int mm = 0, unused = 0;
        const uint32_t H1 = segment_hist<true>(r1 + c.off4[k], c.chunks[k], occ5, s2, mm);
        const uint32_t H2 = segment_hist<false>(r2 + c.off4[k], c.chunks[k], occ5, 0u, unused);
        h1[k] = H1;
        h2[k] = H2;
        m[k] = mm;
        int u[T];
        delta_vector<T>(H1, H2, mm, a, b, u);
        double e = 0.0;
#pragma unroll
        for (int i = 0; i < T; ++i) {
            const int sai = (i == a) - (i == b);
#pragma unroll
            for (int j = 0; j < T; ++j) {
                const int saj = (j == a) - (j == b);
                const int idx = (k * T + i) * T + j;
                const int cp = cnt[idx] + sai * u[j] + saj * u[i];
                const double d = __fma_rn(-(double)cp, c.R[idx], c.E[idx]);
                e = __fma_rn(d, d, e);
            }
        }
        f2 = __fma_rn(c.w[k], e, f2);
    }
    return f2;
}

// Two attempts per Philox call: (x0, x1) then (x2, x3); valid when both draws
// accept and the species differ (pyhea/cpp/accelerate.cpp:649-655).
__device__ __forceinline__ bool draw_pair(const SearchConst &c, uint32_t stream, uint32_t round, uint32_t task,
                                          const uint8_t *occ5, uint32_t &s1, uint32_t &s2)
{
    const uint32_t n = (uint32_t)c.num_sites;
    for (uint32_t call = 0; call < kPhiloxCallsPerDraw; ++call) {
        const u32x4 x = philox4x32_10(u32x4{call, task, round, stream}, c.key0, c.key1);
        uint32_t u, v;
        if (bounded_draw(x.x, n, c.reject_below, u) && bounded_draw(x.y, n, c.reject_below, v) && occ5[u] != occ5[v]) {
            s1 = u;
            s2 = v;
            return true;
        }
        if (bounded_draw(x.z, n, c.reject_below, u) && bounded_draw(x.w, n, c.reject_below, v) && occ5[u] != occ5[v]) {
            s1 = u;
            s2 = v;
            return true;
        }
    }
    return false;
}

__device__ __forceinline__ double inf_d() { return __longlong_as_double(0x7FF0000000000000LL); }

// Lexicographic (f2, task) minimum: the lowest task wins ties.
__device__ __forceinline__ bool better(double f, int q, double bf, int bq) { return f < bf || (f == bf && q < bq); }

__device__ __forceinline__ void warp_argmin(double &f, int &q)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const double of = __shfl_xor_sync(0xFFFFFFFFu, f, o);
        const int oq = __shfl_xor_sync(0xFFFFFFFFu, q, o);
        if (better(of, oq, f, q)) {
            f = of;
            q = oq;
        }
    }
}

// ---------------------------------------------------------------------------
// Block recount of the pair counts of the occupancy in shared memory.
// Per-thread packed 10-bit accumulators [T][S], flushed to shared-memory bins
// every 32 sites (32 sites * 28 entries < 1024).  Sentinel entries land in
// field 0 and are removed at the end (pad_k * n_i per row i).
// ---------------------------------------------------------------------------
template <int T, int S>
__device__ void block_recount(const SearchConst &c, const int4 *__restrict__ nbor, const uint8_t *occ5, int32_t *cnt)
{
    for (int x = threadIdx.x; x < S * T * T; x += blockDim.x) cnt[x] = 0;
    __syncthreads();
    uint64_t acc[T][S];
#pragma unroll
    for (int i = 0; i < T; ++i)
#pragma unroll
        for (int k = 0; k < S; ++k) acc[i][k] = 0;
    auto flush = [&]() {
#pragma unroll
        for (int i = 0; i < T; ++i)
#pragma unroll
            for (int k = 0; k < S; ++k) {
#pragma unroll
                for (int t = 0; t < T; ++t) {
                    const int v = (int)((acc[i][k] >> (10 * t)) & 1023u);
                    if (v) atomicAdd(&cnt[(k * T + i) * T + t], v);
                }
                acc[i][k] = 0;
            }
    };
    int since = 0;
    for (int s = threadIdx.x; s < c.num_sites; s += blockDim.x) {
        const int a5 = occ5[s];
        const int4 *row = nbor + (size_t)s * c.row4;
#pragma unroll
        for (int k = 0; k < S; ++k) {
            uint64_t h = 0;
            const int4 *seg = row + c.off4[k];
            for (int ch = 0; ch < c.chunks[k]; ++ch) {
                const int4 x = __ldg(seg + ch);
                h += (1ull << (2 * occ5[x.x])) + (1ull << (2 * occ5[x.y])) + (1ull << (2 * occ5[x.z])) +
                     (1ull << (2 * occ5[x.w]));
            }
#pragma unroll
            for (int i = 0; i < T; ++i)
                if (a5 == 5 * i) acc[i][k] += h;
        }
        if (++since == 32) {
            flush();
            since = 0;
        }
    }
    flush();
    __syncthreads();
    for (int x = threadIdx.x; x < S * T; x += blockDim.x) {
        const int k = x / T, i = x % T;
        cnt[(k * T + i) * T] -= c.pad[k] * (c.prefix[i + 1] - c.prefix[i]);
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// New random occupancy (keyed Feistel permutation of the sorted layout) or a
// recount of a stored one; writes occupancy, counts and f2 of the slot.
// One CTA per slot; dynamic shared memory = occ_stride + 16 + 4*S*T*T bytes.
// ---------------------------------------------------------------------------
template <int T, int S>
__global__ void __launch_bounds__(512, 1) generate_kernel(const SearchConst c, const GenArgs g)
{
    extern __shared__ __align__(16) uint8_t smem[];
    uint8_t *occ5 = smem;
    int32_t *cnt = reinterpret_cast<int32_t *>(smem + c.occ_stride + 16);
    const int slot = g.order[blockIdx.x];
    uint8_t *gocc = g.occ + (size_t)slot * c.occ_stride;
    const int n = c.num_sites;
    if (g.generate) {
        uint32_t rk[kFeistelRounds];
        const u32x4 w0 = philox4x32_10(u32x4{blockIdx.x, g.generation, 0u, kInitStream}, c.key0, c.key1);
        const u32x4 w1 = philox4x32_10(u32x4{blockIdx.x, g.generation, 1u, kInitStream}, c.key0, c.key1);
        rk[0] = w0.x; rk[1] = w0.y; rk[2] = w0.z; rk[3] = w0.w; rk[4] = w1.x; rk[5] = w1.y;
        for (int s = threadIdx.x; s < n; s += blockDim.x) {
            uint32_t y = feistel((uint32_t)s, c.feistel_h, rk);
            while (y >= (uint32_t)n) y = feistel(y, c.feistel_h, rk);
            int t = 0;
#pragma unroll
            for (int i = 1; i < T; ++i) t += (int)(y >= (uint32_t)c.prefix[i]);
            occ5[s] = (uint8_t)(5 * t);
            gocc[s] = (uint8_t)t;
        }
    } else {
        for (int s = threadIdx.x; s < n; s += blockDim.x) occ5[s] = (uint8_t)(5 * gocc[s]);
    }
    if (threadIdx.x == 0) occ5[n] = 0;
    __syncthreads();
    block_recount<T, S>(c, g.nbor, occ5, cnt);
    int32_t *gc = g.cnt + (size_t)slot * S * T * T;
    for (int x = threadIdx.x; x < S * T * T; x += blockDim.x) gc[x] = cnt[x];
    if (threadIdx.x == 0) g.f2[slot] = fitness_of_counts<T, S>(c, cnt);
}

// ---------------------------------------------------------------------------
// The local parallel search (pyhea/cpp/accelerate.cpp:601-694): one CTA per
// solution, one thread per task (threads loop when tasks > blockDim).  Each
// round every task scores one proposal against the same state; the block takes
// the (f2, task) minimum and accepts it iff it is strictly below the current
// f2; the search ends after `depth` rounds in a row without an accept.
// Dynamic shared memory = occ_stride + 16 + 4*S*T*T + 32*(8+4) + 16 bytes.
// ---------------------------------------------------------------------------
template <int T, int S>
__global__ void __launch_bounds__(512, 1) mc_kernel(const SearchConst c, const McArgs g)
{
    extern __shared__ __align__(16) uint8_t smem[];
    uint8_t *occ5 = smem;
    int32_t *cnt = reinterpret_cast<int32_t *>(smem + c.occ_stride + 16);
    double *red_f = reinterpret_cast<double *>(cnt + ((S * T * T + 3) & ~3));
    int *red_q = reinterpret_cast<int *>(red_f + 32);
    double *ctl_f = reinterpret_cast<double *>(red_q + 32);
    int *ctl_q = reinterpret_cast<int *>(ctl_f + 1);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    const int slot = g.order[blockIdx.x];
    const uint32_t stream = (g.mc_call << 16) | (uint32_t)blockIdx.x;
    uint8_t *gocc = g.occ + (size_t)slot * c.occ_stride;
    int32_t *gcnt = g.cnt + (size_t)slot * S * T * T;
    const int n = c.num_sites;

    {  // stage the slot: occupancy as 5*species (16-byte vectors), counts
        const uint4 *src = reinterpret_cast<const uint4 *>(gocc);
        uint4 *dst = reinterpret_cast<uint4 *>(occ5);
        for (int v = tid; v < c.occ_stride / 16; v += blockDim.x) {
            uint4 x = src[v];
            // bytes are species < 8: 5*t per byte without carries
            x.x = x.x * 5u; x.y = x.y * 5u; x.z = x.z * 5u; x.w = x.w * 5u;
            dst[v] = x;
        }
        for (int x = tid; x < S * T * T; x += blockDim.x) cnt[x] = gcnt[x];
    }
    __syncthreads();
    if (tid == 0) occ5[n] = 0;  // sentinel (occ_stride may end exactly at n)
    __syncthreads();

    double cur = g.f2[slot];
    int miss = 0;
    int64_t round = 0, accepts = 0, evals = 0;
    while (miss < g.depth && round < g.max_rounds) {
        double bf = inf_d();  // +inf
        int bq = 0x7FFFFFFF;
        uint32_t b1 = 0, b2 = 0, bh1[S], bh2[S];
        int bm[S];
        for (int q = tid; q < g.tasks; q += blockDim.x) {
            uint32_t s1, s2;
            if (!draw_pair(c, stream, (uint32_t)round, (uint32_t)q, occ5, s1, s2)) continue;
            ++evals;
            uint32_t h1[S], h2[S];
            int m[S];
            const double f = score_swap<T, S>(c, g.nbor, occ5, cnt, s1, s2, occ5[s1] / 5, occ5[s2] / 5, h1, h2, m);
            if (f < bf) {
                bf = f;
                bq = q;
                b1 = s1;
                b2 = s2;
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    bh1[k] = h1[k];
                    bh2[k] = h2[k];
                    bm[k] = m[k];
                }
            }
        }
        double wf = bf;
        int wq = bq;
        warp_argmin(wf, wq);
        if (lane == 0) {
            red_f[warp] = wf;
            red_q[warp] = wq;
        }
        __syncthreads();
        if (warp == 0) {
            double xf = lane < nwarps ? red_f[lane] : inf_d();
            int xq = lane < nwarps ? red_q[lane] : 0x7FFFFFFF;
            warp_argmin(xf, xq);
            if (lane == 0) {
                *ctl_f = xf;
                *ctl_q = xq;
            }
        }
        __syncthreads();
        const double win_f = *ctl_f;
        const int win_q = *ctl_q;
        if (win_f < cur) {
            if (bq == win_q) {  // this thread owns the winning proposal
                const int a = occ5[b1] / 5, b = occ5[b2] / 5;
                const uint8_t t = occ5[b1];
                occ5[b1] = occ5[b2];
                occ5[b2] = t;
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    int u[T];
                    delta_vector<T>(bh1[k], bh2[k], bm[k], a, b, u);
#pragma unroll
                    for (int j = 0; j < T; ++j) {
                        cnt[(k * T + a) * T + j] += u[j];
                        cnt[(k * T + j) * T + a] += u[j];
                        cnt[(k * T + b) * T + j] -= u[j];
                        cnt[(k * T + j) * T + b] -= u[j];
                    }
                }
                if (g.trace && accepts < g.trace_cap) {
                    AcceptRecord r;
                    r.round = (uint32_t)round;
                    r.task = (uint32_t)win_q;
                    r.s1 = b1;
                    r.s2 = b2;
                    r.f2 = win_f;
                    g.trace[(size_t)blockIdx.x * g.trace_cap + accepts] = r;
                    if (g.trace_counts) {
                        int32_t *dst = g.trace_counts + ((size_t)blockIdx.x * g.trace_cap + accepts) * S * T * T;
                        for (int x = 0; x < S * T * T; ++x) dst[x] = cnt[x];
                    }
                }
            }
            cur = win_f;
            miss = 0;
            ++accepts;
            __syncthreads();
        } else {
            ++miss;
        }
        ++round;
    }

    // write the slot back
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(occ5);
        uint4 *dst = reinterpret_cast<uint4 *>(gocc);
        for (int v = tid; v < c.occ_stride / 16; v += blockDim.x) {
            uint4 x = src[v];
            // every byte holds 5*t with t < 8: t = (5t * 205) >> 10 per byte
            uint32_t o[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                uint32_t r = 0;
#pragma unroll
                for (int by = 0; by < 4; ++by) {
                    const uint32_t b5 = (o[w] >> (8 * by)) & 0xFFu;
                    r |= ((b5 * 205u) >> 10) << (8 * by);
                }
                o[w] = r;
            }
            dst[v] = make_uint4(o[0], o[1], o[2], o[3]);
        }
        for (int x = tid; x < S * T * T; x += blockDim.x) gcnt[x] = cnt[x];
    }
    // evals per thread -> block total
    unsigned long long ev = (unsigned long long)evals;
#pragma unroll
    for (int o = 16; o; o >>= 1) ev += __shfl_xor_sync(0xFFFFFFFFu, ev, o);
    if (lane == 0 && ev) atomicAdd(&g.stats[1], ev);
    if (tid == 0) {
        g.f2[slot] = cur;
        atomicAdd(&g.stats[0], (unsigned long long)round);
        atomicAdd(&g.stats[2], (unsigned long long)accepts);
        if (g.trace_len) g.trace_len[blockIdx.x] = accepts;
        if (g.rounds_out) g.rounds_out[blockIdx.x] = round;
    }
}

// ---------------------------------------------------------------------------
// Stable ordering of populations by f2 (pyhea/cpp/accelerate.cpp:37-64,
// :305-330): rank_i = #{j : f_j < f_i} + #{j < i : f_j == f_i}; order is
// rewritten in rank order.  One CTA; `count` <= 2 * 65535.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) sort_slots_kernel(int32_t *order, const double *f2, int count, int32_t *scratch)
{
    for (int i = threadIdx.x; i < count; i += blockDim.x) scratch[i] = order[i];
    __syncthreads();
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
        const double fi = f2[scratch[i]];
        int r = 0;
        for (int j = 0; j < count; ++j) {
            const double fj = f2[scratch[j]];
            r += (fj < fi) || (fj == fi && j < i);
        }
        order[r] = scratch[i];
    }
}

}  // namespace hea
