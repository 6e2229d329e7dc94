// hea_search.cuh -- the swap-search kernels (sm_100a), templated on the number
// of species T and on the shell layout of the neighbour table.
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
#include <utility>

#include "hea_device.cuh"

namespace hea {

// Implicit neighbour ids of a perfect FCC/BCC cube (the structure keeps no
// neighbour table in memory).  Site s = nb (cx L^2 + cy L + cz) + b is basis
// site b of cell (cx, cy, cz).  Its neighbours (shells concatenated) lie in
// cells (cx + dx, cy + dy, cz + dz), d in {-1, 0, 1}, periodic in every axis,
// at basis b' -- both fixed by the lattice's shell vectors.  Shell generators
// in half lattice units: FCC (1,1,0) 12, (2,0,0) 6, then (2,2,0) 12 (reference
// set) or (2,1,1) 24 (true third shell); BCC (1,1,1) 8, (2,0,0) 6, (2,2,0) 12.
// The sets equal the table of pyhea/lattice/lattice.py:196-323; entries of a
// shell come in another order, which no count or histogram sees.
struct LatticeConst {
    int32_t L;                   // cube edge in cells; 0: the structure has a neighbour table
    int32_t nb;                  // basis sites per cell (4 FCC, 2 BCC)
    int32_t zsize[3], zoff[3];   // shell sizes and offsets in the concatenated neighbour list
    double inv_L, inv_LL;        // 1 / L and 1 / L^2, rounded (lattice_cell)
    int32_t kind;                // kLatFccRef, kLatFccTrue3 or kLatBcc
    int32_t pad_;
};
static_assert(sizeof(LatticeConst) % 8 == 0, "LatticeConst keeps SearchConst 8-byte sized");

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
    uint32_t draw16;    // 1: 16-bit draws, four attempts per Philox call (use_draw16)
    uint32_t reject16;  // 2^16 mod N
    uint32_t hist_stream;  // 1: site histograms read with streaming (evict-first) loads (load_hist)
    uint32_t pad_;
    LatticeConst lat;   // lat.L > 0: neighbours from lattice arithmetic (nbor unused)
};

enum : int { kLatFccRef = 0, kLatFccTrue3 = 1, kLatBcc = 2 };

__host__ __device__ constexpr int lat_nb(int kind) { return kind == kLatBcc ? 2 : 4; }
__host__ __device__ constexpr int lat_basis(int kind, int b, int d)
{
    // half-unit basis offsets: FCC {0,0,0} {1,1,0} {1,0,1} {0,1,1}; BCC {0,0,0} {1,1,1}
    return kind == kLatBcc ? b : (b == 0 ? 0 : (d == 0 ? (b != 3) : d == 1 ? (b != 2) : (b != 1)));
}
__host__ __device__ constexpr int lat_gen(int kind, int k, int d)
{
    return k == 0 ? (kind == kLatBcc ? 1 : (d < 2 ? 1 : 0))
         : k == 1 ? (d == 0 ? 2 : 0)
         : (kind == kLatFccTrue3 ? (d == 0 ? 2 : 1) : (d < 2 ? 2 : 0));
}
__host__ __device__ constexpr int lat_shell_size(int kind, int k)
{
    return k == 0 ? (kind == kLatBcc ? 8 : 12) : k == 1 ? 6 : (kind == kLatFccTrue3 ? 24 : 12);
}

// The distinct signed axis permutations of shell k's generator, in a fixed order.
struct LatVecs {
    int n;
    int v[24][3];
};
__host__ __device__ constexpr LatVecs lat_vecs(int kind, int k)
{
    LatVecs out{};
    const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    for (int i = 0; i < 48; ++i) {
        int c[3] = {0, 0, 0};
        for (int d = 0; d < 3; ++d) c[d] = (((i >> (2 - d)) & 1) ? -1 : 1) * lat_gen(kind, k, perm[i >> 3][d]);
        bool dup = false;
        for (int j = 0; j < out.n && !dup; ++j) dup = out.v[j][0] == c[0] && out.v[j][1] == c[1] && out.v[j][2] == c[2];
        if (!dup) {
            for (int d = 0; d < 3; ++d) out.v[out.n][d] = c[d];
            ++out.n;
        }
    }
    return out;
}
// Packed neighbour descriptor for basis b and offset v: (dx+1) | (dy+1) << 2 | (dz+1) << 4 | b' << 6.
__host__ __device__ constexpr int lat_pack(int kind, int b, const int (&v)[3])
{
    int out = 0, par[3] = {0, 0, 0};
    for (int d = 0; d < 3; ++d) {
        const int q = lat_basis(kind, b, d) + v[d];  // -2 .. 3 half units
        par[d] = q & 1;
        out |= ((q >= 0 ? q / 2 : -1) + 1) << (2 * d);
    }
    int bp = 0;
    for (int x = 0; x < lat_nb(kind); ++x)
        if (lat_basis(kind, x, 0) == par[0] && lat_basis(kind, x, 1) == par[1] && lat_basis(kind, x, 2) == par[2])
            bp = x;
    return out | (bp << 6);
}
__host__ __device__ constexpr int lat_desc(int kind, int b, int k, int e) { return lat_pack(kind, b, lat_vecs(kind, k).v[e]); }

// Every descriptor, shells concatenated, for the per-lane lookups of
// lattice_neighbor (a global table: lanes read different entries, which the
// constant bank would serialise).
struct LatDescTable {
    uint8_t d[3][4][54];
};
__host__ __device__ constexpr LatDescTable make_lat_desc_table()
{
    LatDescTable t{};
    for (int kind = 0; kind < 3; ++kind) {
        int e0 = 0;
        for (int k = 0; k < 3; ++k) {
            const LatVecs vs = lat_vecs(kind, k);
            for (int b = 0; b < lat_nb(kind); ++b)
                for (int e = 0; e < vs.n; ++e) t.d[kind][b][e0 + e] = (uint8_t)lat_pack(kind, b, vs.v[e]);
            e0 += vs.n;
        }
    }
    return t;
}
__device__ const LatDescTable kLatDesc = make_lat_desc_table();

// floor(n / d) for 0 <= n < 2^31, d <= 2^20, from inv = 1/d rounded: n * inv is
// within 2^-21 of n / d, so the truncation is the quotient or one less, and
// one correction makes it exact.
__device__ __forceinline__ int div_by(int n, int d, double inv)
{
    int q = __double2int_rz(__dmul_rn((double)n, inv));
    q += (n - q * d) >= d;
    return q;
}

struct LatticeCell {
    int b, x, y, z;
};

__device__ __forceinline__ LatticeCell lattice_cell(const LatticeConst &lc, int s)
{
    const int cell = s >> (lc.nb == 4 ? 2 : 1), LL = lc.L * lc.L;  // nb is 2 or 4
    const int x = div_by(cell, LL, lc.inv_LL), r = cell - x * LL, y = div_by(r, lc.L, lc.inv_L);
    return LatticeCell{s & (lc.nb - 1), x, y, r - y * lc.L};
}

// Entry e (shells concatenated) of the neighbour list of the site in cell p.
__device__ __forceinline__ int lattice_neighbor(const LatticeConst &lc, const LatticeCell &p, int e)
{
    const int d = __ldg(&kLatDesc.d[lc.kind][p.b][e]), L = lc.L;
    int x = p.x + (d & 3) - 1, y = p.y + ((d >> 2) & 3) - 1, z = p.z + ((d >> 4) & 3) - 1;
    x += x < 0 ? L : 0;
    y += y < 0 ? L : 0;
    z += z < 0 ? L : 0;
    x -= x >= L ? L : 0;
    y -= y >= L ? L : 0;
    z -= z >= L ? L : 0;
    return lc.nb * ((x * L + y) * L + z) + (d >> 6);
}

// How often s2 is listed in each of the first S shells of s1's neighbour
// list, in closed form: the displacement from s1 to s2 in half units, wrapped
// to (-L, L] per axis, is a shell vector iff its absolute components form the
// shell's pattern (FCC 1,1,0 | 2,0,0 | 2,2,0 or 2,1,1; BCC 1,1,1 | 2,0,0 |
// 2,2,0).  At L = 2 the vectors +2 and -2 along an axis reach the same site,
// so each such component doubles the count.  s1 != s2.
template <int S>
__device__ __forceinline__ void lattice_multiplicity(const LatticeConst &lc, int s1, int s2, uint32_t (&m)[S])
{
    const LatticeCell p = lattice_cell(lc, s1), q = lattice_cell(lc, s2);
    const int M = 2 * lc.L, pc[3] = {p.x, p.y, p.z}, qc[3] = {q.x, q.y, q.z};
    int n0 = 0, n1 = 0, n2 = 0, mult = 1;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        int v = 2 * (qc[d] - pc[d]) + lat_basis(lc.kind, q.b, d) - lat_basis(lc.kind, p.b, d);  // (-2L, 2L)
        v -= v > lc.L ? M : 0;
        v += v <= -lc.L ? M : 0;
        const int a = v < 0 ? -v : v;
        n0 += a == 0;
        n1 += a == 1;
        n2 += a == 2;
        mult <<= (M == 4 && a == 2) ? 1 : 0;
    }
    const bool bcc = lc.kind == kLatBcc, true3 = lc.kind == kLatFccTrue3;
    const bool in[3] = {bcc ? n1 == 3 : (n1 == 2 && n0 == 1), n2 == 1 && n0 == 2,
                        true3 ? (n2 == 1 && n1 == 2) : (n2 == 2 && n0 == 1)};
#pragma unroll
    for (int k = 0; k < S; ++k) m[k] = in[k] ? (uint32_t)mult : 0u;
}

// Compile-time form of the same geometry for the walks over every site
// (recounts): with (kind, b, shell, entry) known at compile time a
// neighbour's id is one sum of three per-site axis terms (LatticeAxes) and b'.
// Per-site axis terms: x[d] = nb L^2 wrap(cx + d - 1), y[d] = nb L wrap(cy + d - 1), z[d] = nb wrap(cz + d - 1).
struct LatticeAxes {
    int x[3], y[3], z[3];
};

__device__ __forceinline__ LatticeAxes lattice_axes(int L, int nb, int cx, int cy, int cz)
{
    const int sx = nb * L * L, sy = nb * L;
    LatticeAxes a;
    a.x[0] = (cx == 0 ? L - 1 : cx - 1) * sx;
    a.x[1] = cx * sx;
    a.x[2] = (cx == L - 1 ? 0 : cx + 1) * sx;
    a.y[0] = (cy == 0 ? L - 1 : cy - 1) * sy;
    a.y[1] = cy * sy;
    a.y[2] = (cy == L - 1 ? 0 : cy + 1) * sy;
    a.z[0] = (cz == 0 ? L - 1 : cz - 1) * nb;
    a.z[1] = cz * nb;
    a.z[2] = (cz == L - 1 ? 0 : cz + 1) * nb;
    return a;
}

template <int D>
__device__ __forceinline__ int lat_id(const LatticeAxes &a)
{
    return a.x[D & 3] + a.y[(D >> 2) & 3] + a.z[(D >> 4) & 3] + (D >> 6);
}

template <int Kind, int B, int K, class H, class W, int... E>
__device__ __forceinline__ H lat_shell_sum(const LatticeAxes &a, W &weight, std::integer_sequence<int, E...>)
{
    return (H(0) + ... + weight(lat_id<lat_desc(Kind, B, K, E)>(a)));
}

// Cells first, first + stride, ... of basis B: site(s, h) with h[k] = sum of
// weight(n) over the shell-k neighbours n of site s.
template <int Kind, int B, int S, class H, class W, class F>
__device__ __forceinline__ void lattice_walk(int L, int first, int stride, W &weight, F &site)
{
    constexpr int NB = lat_nb(Kind);
    const int LL = L * L, ncell = LL * L;
    int cell = first;
    int cx = cell / LL, cy = (cell - cx * LL) / L, cz = cell - cx * LL - cy * L;
    const int bx = stride / LL, by = (stride - bx * LL) / L, bz = stride - bx * LL - by * L;
    for (; cell < ncell; cell += stride) {
        const LatticeAxes a = lattice_axes(L, NB, cx, cy, cz);
        H h[S];
        h[0] = lat_shell_sum<Kind, B, 0, H>(a, weight, std::make_integer_sequence<int, lat_shell_size(Kind, 0)>{});
        if constexpr (S > 1)
            h[1] = lat_shell_sum<Kind, B, 1, H>(a, weight, std::make_integer_sequence<int, lat_shell_size(Kind, 1)>{});
        if constexpr (S > 2)
            h[2] = lat_shell_sum<Kind, B, 2, H>(a, weight, std::make_integer_sequence<int, lat_shell_size(Kind, 2)>{});
        site(NB * cell + B, h);
        cz += bz;  // next cell of the walk: cell += stride in (cx, cy, cz) digits
        if (cz >= L) {
            cz -= L;
            ++cy;
        }
        cy += by;
        if (cy >= L) {
            cy -= L;
            ++cx;
        }
        cx += bx;
    }
}

// Every site of an implicit lattice (this thread's share of a walk that
// starts at cell `first` and steps by `stride` cells, once per basis index, so
// that the threads of a warp share the basis and the neighbour geometry is
// compile-time): site(s, h[S]) with h[k] = sum of weight(n) over the shell-k
// neighbours n of s.
template <int S, class H, class W, class F>
__device__ __forceinline__ void lattice_sites(const LatticeConst &lc, int first, int stride, W weight, F site)
{
    if (lc.kind == kLatBcc) {
        lattice_walk<kLatBcc, 0, S, H>(lc.L, first, stride, weight, site);
        lattice_walk<kLatBcc, 1, S, H>(lc.L, first, stride, weight, site);
    } else if (lc.kind == kLatFccTrue3) {
        lattice_walk<kLatFccTrue3, 0, S, H>(lc.L, first, stride, weight, site);
        lattice_walk<kLatFccTrue3, 1, S, H>(lc.L, first, stride, weight, site);
        lattice_walk<kLatFccTrue3, 2, S, H>(lc.L, first, stride, weight, site);
        lattice_walk<kLatFccTrue3, 3, S, H>(lc.L, first, stride, weight, site);
    } else {
        lattice_walk<kLatFccRef, 0, S, H>(lc.L, first, stride, weight, site);
        lattice_walk<kLatFccRef, 1, S, H>(lc.L, first, stride, weight, site);
        lattice_walk<kLatFccRef, 2, S, H>(lc.L, first, stride, weight, site);
        lattice_walk<kLatFccRef, 3, S, H>(lc.L, first, stride, weight, site);
    }
}

// Shell layout of the padded table, in int4 chunks per shell (0: shell absent).
// Fixed layouts unroll every load; RuntimeShells reads the chunk counts from
// SearchConst; ImplicitShells has no table (neighbours from lattice
// arithmetic), so the search loops of table structures carry no implicit
// code and the other way round.
template <int C0, int C1, int C2>
struct Shells {
    static constexpr int S = (C0 > 0) + (C1 > 0) + (C2 > 0);
    static constexpr bool kRuntime = false;
    static constexpr bool kImplicit = false;
    static constexpr int kRow4 = C0 + C1 + C2;
    __host__ __device__ static constexpr int chunks(int k) { return k == 0 ? C0 : (k == 1 ? C1 : C2); }
    __host__ __device__ static constexpr int off(int k) { return k == 0 ? 0 : (k == 1 ? C0 : C0 + C1); }
};
template <int S_>
struct RuntimeShells {
    static constexpr int S = S_;
    static constexpr bool kRuntime = true;
    static constexpr bool kImplicit = false;
    static constexpr int kRow4 = 0;
    __host__ __device__ static constexpr int chunks(int) { return 0; }
    __host__ __device__ static constexpr int off(int) { return 0; }
};
template <int S_>
struct ImplicitShells {
    static constexpr int S = S_;
    static constexpr bool kRuntime = true;
    static constexpr bool kImplicit = true;
    static constexpr int kRow4 = 0;
    __host__ __device__ static constexpr int chunks(int) { return 0; }
    __host__ __device__ static constexpr int off(int) { return 0; }
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
    uint4 *hist;              // [slots][N] site histograms (see block_recount)
    const uint32_t *nbmask;   // neighbour-offset bitmap (see score_swap_hist)
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
    uint4 *hist;  // [slots][N] site histograms written by the recount (nullptr: none)
    const int32_t *order;
    uint32_t generation;
    int32_t generate;  // 1: draw a new occupancy; 0: recount the stored one
};

// ---------------------------------------------------------------------------
// Fitness: f2 = sum_k w_k e_k; e_k accumulates d^2 with fma over the upper
// triangle row by row (d_ii, then d_ij and d_ji for j > i); d = fma(-C', R, E).
// Counts are symmetric and R_ij == R_ji, so d_ij and d_ji share C' and R.
// ---------------------------------------------------------------------------
template <int T, int S>
__device__ __forceinline__ double fitness_of_counts(const SearchConst &c, const int32_t *cnt)
{
    double f2 = 0.0;
#pragma unroll
    for (int k = 0; k < S; ++k) {
        double e = 0.0;
#pragma unroll
        for (int i = 0; i < T; ++i) {
            const int ii = (k * T + i) * T + i;
            const double dii = __fma_rn(-(double)cnt[ii], c.R[ii], c.E[ii]);
            e = __fma_rn(dii, dii, e);
#pragma unroll
            for (int j = i + 1; j < T; ++j) {
                const int ij = (k * T + i) * T + j, ji = (k * T + j) * T + i;
                const double cp = (double)cnt[ij];
                const double dij = __fma_rn(-cp, c.R[ij], c.E[ij]);
                const double dji = __fma_rn(-cp, c.R[ij], c.E[ji]);
                e = __fma_rn(dij, dij, e);
                e = __fma_rn(dji, dji, e);
            }
        }
        f2 = __fma_rn(c.w[k], e, f2);
    }
    return f2;
}

// ---------------------------------------------------------------------------
// The swap delta (how proposals are scored).  Swapping species a (at s1) and b
// (at s2) changes the pair counts of shell k by dC_ij = sa_i u_j + sa_j u_i,
// sa = e_a - e_b, where u_t = n2_t - n1_t + m ([t = b] - [t = a]); n1, n2 are
// the species histograms of the two sites' shell-k neighbourhoods and m is how
// often s2 is listed among s1's shell-k neighbours.  dC is zero outside rows and
// columns a, b, so with d = E - R C (R symmetric) the change of
// e_k = sum_ij d_ij^2 is exactly
//     sum_t u_t (L_t + u_t Q_t) + (u_a - u_b)^2 Cq,
//     L_t = -2 (G_at - G_bt),   G_it = R_it (d_it + d_ti),
//     Q_t = 2 (R_at^2 + R_bt^2) for t != a, b,   Q_a = 4 R_aa^2,   Q_b = 4 R_bb^2,
//     Cq  = 2 R_ab^2,
// and f2 changes by D = sum_k w_k (that).  Each search keeps, per shell k and
// ordered pair (a, b), the row {w L_t, w Q_t} (t < T), {w Cq, 0} in shared
// memory (the delta table; Q and Cq depend on the structure only, L on the
// counts and is rebuilt after every accepted swap) and scores a proposal by D
// alone: O(T) terms per shell instead of the O(T^2) of a full fitness.
// Fixed operation order (restated by the CPU oracle):
//     Q   = w * (2 * (R_at * R_at + R_bt * R_bt)),  Q_a = w * (4 * (R_aa * R_aa)),
//     Cq  = w * (2 * (R_ab * R_ab)),
//     d_it = fma(-C, R_it, E_it),  G_it = R_it * (d_it + d_ti),  L = (-2 * w) * (G_at - G_bt),
//     D = 0; per shell k: per t < T: D = fma(u_t, fma(u_t, Q_t, L_t), D); then D = fma((u_a - u_b)^2, Cq, D).
// A round's best proposal (lowest D, lowest task on ties) is accepted iff D < 0;
// the search's running f2 adds D, and the f2 a search stores at its end is
// recomputed from the counts (fitness_of_counts).
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int delta_row(int T) { return (T + 1) | 1; }  // odd: lanes' rows spread over the banks
__host__ __device__ constexpr int delta_entries(int T, int S) { return S * T * T * delta_row(T); }  // double2 entries

// Structure constants of the table: w Q_t in .y of entries t < T, w Cq in .x
// of entry T, for every (k, a, b), a != b.  Block-cooperative, no barrier.
template <int T, int S>
__device__ void delta_consts(const SearchConst &c, double2 *tab)
{
    constexpr int R = delta_row(T);
    for (int e = threadIdx.x; e < S * T * T * R; e += blockDim.x) {
        const int t = e % R, ab = (e / R) % (T * T), k = e / (R * T * T);
        const int a = ab / T, b = ab % T;
        if (a == b || t > T) continue;
        const double *Rk = c.R + k * T * T;
        const double w = c.w[k];
        if (t == T) {
            tab[e].x = __dmul_rn(w, __dmul_rn(2.0, __dmul_rn(Rk[a * T + b], Rk[a * T + b])));
        } else if (t == a || t == b) {
            tab[e].y = __dmul_rn(w, __dmul_rn(4.0, __dmul_rn(Rk[t * T + t], Rk[t * T + t])));
        } else {
            const double p = __dmul_rn(Rk[a * T + t], Rk[a * T + t]), q = __dmul_rn(Rk[b * T + t], Rk[b * T + t]);
            tab[e].y = __dmul_rn(w, __dmul_rn(2.0, __dadd_rn(p, q)));
        }
    }
}

// The count-dependent half of the table: w L_t in .x of entries t < T, from
// the counts count_of(k, i, j) (symmetric in i, j).  Groups of T lanes of a
// warp hold G_xt for x = 0..T-1 of one (shell, t); each lane takes the others'
// G by shuffle and writes its row x against every y != x.  Warps call it
// convergently (full-mask shuffles); no barrier inside.
template <int T, int S, class CountOf>
__device__ __forceinline__ void delta_linear(const SearchConst &c, double2 *tab, CountOf count_of)
{
    constexpr int R = delta_row(T), kGroups = 32 / T, kWarps = (S * T + kGroups - 1) / kGroups;
    const int lane = threadIdx.x & 31, x = lane % T, grp = lane / T;
    for (int w = threadIdx.x >> 5; w < kWarps; w += blockDim.x >> 5) {
        const int g = w * kGroups + grp;  // shell k = g / T, column t = g % T
        const bool on = grp < kGroups && g < S * T;
        const int k = on ? g / T : 0, t = on ? g % T : 0;
        const int xt = (k * T + x) * T + t, tx = (k * T + t) * T + x;
        double G = 0.0, m2w = 0.0;
        if (on) {
            const double C = (double)count_of(k, x, t);
            const double dxt = __fma_rn(-C, c.R[xt], c.E[xt]);
            const double dtx = __fma_rn(-C, c.R[xt], c.E[tx]);
            G = __dmul_rn(c.R[xt], __dadd_rn(dxt, dtx));
            m2w = __dmul_rn(-2.0, c.w[k]);
        }
#pragma unroll
        for (int y = 0; y < T; ++y) {
            const double Gy = __shfl_sync(0xFFFFFFFFu, G, lane - x + y);
            if (on && y != x) tab[((k * T + x) * T + y) * R + t].x = __dmul_rn(m2w, __dsub_rn(G, Gy));
        }
    }
}

__device__ __forceinline__ int field5(uint32_t h, int shift) { return (int)((h >> shift) & 31u); }

__device__ __forceinline__ int count4(const int4 x, uint32_t v)
{
    return ((uint32_t)x.x == v) + ((uint32_t)x.y == v) + ((uint32_t)x.z == v) + ((uint32_t)x.w == v);
}

// D of one proposal: s1 (species a, site histograms p), s2 (b, q).  On return
// h1, h2 are the shell histograms with m folded in -- h1_k + (m << 5a), h2_k +
// (m << 5b) -- so that u_t = field_t(h2_k) - field_t(h1_k); the fields stay
// below 32 (n1_a + m <= Z_k because s1's list holds s2, of species b, m times;
// likewise for h2).  nbmask has bit (n - s + N - 1) set for every table entry n
// of every site s: a clear bit for s2 - s1 proves m = 0 in every shell, a set
// bit sends the lane to count s2 in s1's row.
template <int T, class L>
__device__ __forceinline__ double score_delta(const SearchConst &c, const int4 *__restrict__ nbor,
                                              const uint32_t *__restrict__ nbmask, const double2 *tab, const uint4 p,
                                              const uint4 q, uint32_t s1, uint32_t s2, int a, int b,
                                              uint32_t (&h1)[L::S], uint32_t (&h2)[L::S])
{
    constexpr int S = L::S, R = delta_row(T);
    const uint32_t d = s2 - s1 + (uint32_t)c.num_sites - 1u;
    const bool near = (__ldg(nbmask + (d >> 5)) >> (d & 31u)) & 1u;
    const uint32_t pv[3] = {p.x, p.y, p.z}, qv[3] = {q.x, q.y, q.z};
#pragma unroll
    for (int k = 0; k < S; ++k) {
        h1[k] = pv[k];
        h2[k] = qv[k];
    }
    const int a5 = 5 * a, b5 = 5 * b;
    if (near) {
        if constexpr (L::kImplicit) {
            uint32_t m[S];
            lattice_multiplicity<S>(c.lat, (int)s1, (int)s2, m);
#pragma unroll
            for (int k = 0; k < S; ++k) {
                h1[k] += m[k] << a5;
                h2[k] += m[k] << b5;
            }
        } else {
            const int row4 = L::kRuntime ? c.row4 : L::kRow4;
            const int4 *r1 = nbor + (size_t)s1 * row4;
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const int o = L::kRuntime ? c.off4[k] : L::off(k), n = L::kRuntime ? c.chunks[k] : L::chunks(k);
                uint32_t m = 0;
                for (int ch = 0; ch < n; ++ch) m += count4(__ldg(r1 + o + ch), s2);
                h1[k] += m << a5;
                h2[k] += m << b5;
            }
        }
    }
    const double2 *row = tab + (a * T + b) * R;
    double D = 0.0;
#pragma unroll
    for (int k = 0; k < S; ++k) {
        const double2 *e = row + k * T * T * R;
#pragma unroll
        for (int t = 0; t < T; ++t) {
            const double u = (double)(field5(h2[k], 5 * t) - field5(h1[k], 5 * t));
            const double2 lq = e[t];
            D = __fma_rn(u, __fma_rn(u, lq.y, lq.x), D);
        }
        const int v = field5(h2[k], a5) - field5(h1[k], a5) - field5(h2[k], b5) + field5(h1[k], b5);
        D = __fma_rn((double)(v * v), e[T].x, D);
    }
    return D;
}

// After an accepted swap of s1 (species a -> b) and s2 (b -> a): update the
// histograms of every neighbour listed in both rows (block-wide, atomics in
// L2; the caller's barrier publishes them).  An entry n in shell k of s1's row
// means s1 is in n's shell k as often, since tables are symmetric per shell.
// kSpeciesWord: also the species words of s1 and s2, which draw_pair_hist
// reads; searches whose draws read the occupancy leave them at their recount
// values.
// `me` is this thread's index in the block's order of the work (a rotation of
// threadIdx.x, so that other updates can run on the first warps meanwhile).
template <class L, bool kSpeciesWord>
__device__ __forceinline__ void update_hist(const SearchConst &c, const int4 *__restrict__ nbor, uint4 *hist,
                                            uint32_t s1, uint32_t s2, int a, int b, int me)
{
    const uint32_t up = (1u << (5 * b)) - (1u << (5 * a));  // s1's neighbours: one a becomes b
    if constexpr (L::kImplicit) {  // row e of s1 then of s2, shells concatenated
        const int row = c.lat.zoff[L::S - 1] + c.lat.zsize[L::S - 1];
        for (int e = me; e < 2 * row; e += blockDim.x) {
            const bool first = e < row;
            const int idx = first ? e : e - row;
            const int n = lattice_neighbor(c.lat, lattice_cell(c.lat, (int)(first ? s1 : s2)), idx);
            int k = 0;
#pragma unroll
            for (int kk = 1; kk < L::S; ++kk) k += idx >= c.lat.zoff[kk];
            atomicAdd(reinterpret_cast<uint32_t *>(hist + n) + k, first ? up : 0u - up);
        }
    } else {
    const int row4 = L::kRuntime ? c.row4 : L::kRow4;
    const int row = 4 * row4;
    for (int e = me; e < 2 * row; e += blockDim.x) {
        const bool first = e < row;
        const int idx = first ? e : e - row;
        const int32_t *r = reinterpret_cast<const int32_t *>(nbor + (size_t)(first ? s1 : s2) * row4);
        const int n = __ldg(r + idx);
        if (n >= c.num_sites) continue;  // sentinel padding
        int k = 0;
#pragma unroll
        for (int kk = 1; kk < L::S; ++kk) k += idx >= 4 * (L::kRuntime ? c.off4[kk] : L::off(kk));
        uint32_t *h = reinterpret_cast<uint32_t *>(hist + n) + k;
        atomicAdd(h, first ? up : 0u - up);
    }
    }
    if (kSpeciesWord && me == 0) {
        hist[s1].w = (uint32_t)(5 * b);
        hist[s2].w = (uint32_t)(5 * a);
    }
}

// The three updates of an accepted swap on different warps where the block has
// enough of them: the table's L half on warps [0, delta_linear's warps), the
// new counts on the next warps, the neighbours' histograms after those.  The
// rotated thread indices (block_rotation) keep every loop covering its work once.
template <int T, int S>
__host__ __device__ constexpr int accept_linear_warps() { return (S * T + 32 / T - 1) / (32 / T); }
__device__ __forceinline__ int block_rotation(int by)
{
    int me = (int)threadIdx.x - by;
    while (me < 0) me += blockDim.x;
    return me;
}

// Two attempts per Philox call: (x0, x1) then (x2, x3); valid when both draws
// accept and the species differ (pyhea/cpp/accelerate.cpp:649-655).  With
// 16-bit draws (draw16), four attempts per call: attempt j takes the low and
// the high half of word x_j.  differ(u, v) reads the two sites' species.
template <class Differ>
__device__ __forceinline__ bool draw_pair_by(const SearchConst &c, uint32_t stream, uint32_t round, uint32_t task,
                                             Differ &&differ, uint32_t &s1, uint32_t &s2)
{
    const uint32_t n = (uint32_t)c.num_sites;
    if (c.draw16) {
        for (uint32_t call = 0; call < kPhiloxCallsPerDraw; ++call) {
            const u32x4 x = philox4x32_10(u32x4{call, task, round, stream}, c.key0, c.key1);
            const uint32_t w[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                uint32_t u, v;
                if (bounded_draw16(w[j] & 0xFFFFu, n, c.reject16, u) && bounded_draw16(w[j] >> 16, n, c.reject16, v) &&
                    differ(u, v)) {
                    s1 = u;
                    s2 = v;
                    return true;
                }
            }
        }
        return false;
    }
    for (uint32_t call = 0; call < kPhiloxCallsPerDraw; ++call) {
        const u32x4 x = philox4x32_10(u32x4{call, task, round, stream}, c.key0, c.key1);
        uint32_t u, v;
        if (bounded_draw(x.x, n, c.reject_below, u) && bounded_draw(x.y, n, c.reject_below, v) && differ(u, v)) {
            s1 = u;
            s2 = v;
            return true;
        }
        if (bounded_draw(x.z, n, c.reject_below, u) && bounded_draw(x.w, n, c.reject_below, v) && differ(u, v)) {
            s1 = u;
            s2 = v;
            return true;
        }
    }
    return false;
}

// Species from the occupancy (5*species bytes).
__device__ __forceinline__ bool draw_pair(const SearchConst &c, uint32_t stream, uint32_t round, uint32_t task,
                                          const uint8_t *occ5, uint32_t &s1, uint32_t &s2)
{
    return draw_pair_by(c, stream, round, task, [occ5](uint32_t u, uint32_t v) { return occ5[u] != occ5[v]; }, s1, s2);
}

// One site's histogram entry.  Structures whose histograms are far larger
// than L2 (hist_stream, set by the host) read them with evict-first loads:
// random 16-byte DRAM loads run 1.35x faster that way on B200 and the lines
// they bring do not push out those of structures that do stay in L2; an
// L2-resident structure keeps the default policy (evict-first lost 3 % there).
__device__ __forceinline__ uint4 load_hist(const SearchConst &c, const uint4 *h)
{
    return c.hist_stream ? __ldcs(h) : __ldcg(h);
}

// Species from the site histograms' species words (hist[s].w = 5*species):
// for an occupancy in HBM this makes the two 16-byte L2 loads of an attempt
// the only memory round trip of a proposal; p, q are the accepted pair's
// histograms.
__device__ __forceinline__ bool draw_pair_hist(const SearchConst &c, uint32_t stream, uint32_t round, uint32_t task,
                                               const uint4 *hist, uint32_t &s1, uint32_t &s2, uint4 &p, uint4 &q)
{
    return draw_pair_by(
        c, stream, round, task,
        [&c, hist, &p, &q](uint32_t u, uint32_t v) {
            p = load_hist(c, hist + u);
            q = load_hist(c, hist + v);
            return p.w != q.w;
        },
        s1, s2);
}

// Ordering key of a proposal's delta D: ~bits(D) for D < 0 (more negative,
// smaller key), all ones for a proposal that does not improve (D >= 0) or for
// no proposal.  The round's winner is the lexicographic (key, task) minimum.
constexpr uint64_t kNoSwap = ~0ull;
__device__ __forceinline__ uint64_t delta_key(double D)
{
    return D < 0.0 ? ~(uint64_t)__double_as_longlong(D) : kNoSwap;
}
__device__ __forceinline__ double key_delta(uint64_t key) { return __longlong_as_double((long long)~key); }
__device__ __forceinline__ bool better(uint64_t k, int q, uint64_t bk, int bq) { return k < bk || (k == bk && q < bq); }

// The warp's lexicographic (key, q) minimum in every lane, q >= 0: three
// 32-bit warp reductions (high word, low word among the lanes holding the
// minimal high word, task among the lanes holding the minimal key).
__device__ __forceinline__ void warp_argmin(uint64_t &key, int &q)
{
    const uint32_t hi = (uint32_t)(key >> 32), lo = (uint32_t)key;
    const uint32_t mhi = __reduce_min_sync(0xFFFFFFFFu, hi);
    const uint32_t mlo = __reduce_min_sync(0xFFFFFFFFu, hi == mhi ? lo : 0xFFFFFFFFu);
    const uint32_t mq = __reduce_min_sync(0xFFFFFFFFu, (hi == mhi && lo == mlo) ? (uint32_t)q : 0xFFFFFFFFu);
    key = ((uint64_t)mhi << 32) | mlo;
    q = (int)mq;
}

// Exact site histogram (5-bit field per species) from the recount's 10-bit
// fields, less the sentinel entries the padding added to species 0.
template <int T>
__device__ __forceinline__ uint32_t pack_hist5(uint64_t h10, int pad)
{
    uint32_t r = 0;
#pragma unroll
    for (int t = 0; t < T; ++t) r |= (uint32_t)((h10 >> (10 * t)) & 1023u) << (5 * t);
    return r - (uint32_t)pad;
}

// ---------------------------------------------------------------------------
// Block recount of the pair counts of the occupancy in shared memory.
// With `hist`, also writes every site's histograms: hist[s] = {H_0, H_1, H_2,
// 5 species(s)}, H_k = sum over s's shell-k neighbours n of 1 << (5
// species(n)) -- the species histogram of the neighbourhood, one 5-bit field
// per species -- and the last word the site's own species (5*species).
// Per-thread packed 10-bit accumulators [T][S], flushed to shared-memory bins
// every 32 sites (32 sites * 28 entries < 1024).  Sentinel entries land in
// field 0 and are removed at the end (pad_k * n_i per row i).
// ---------------------------------------------------------------------------
template <int T, int S>
__device__ void block_recount(const SearchConst &c, const int4 *__restrict__ nbor, const uint8_t *occ5, int32_t *cnt,
                              uint4 *hist = nullptr)
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
    // one site with its shell histograms h (10-bit fields)
    const auto site = [&](int s, const uint64_t (&h)[S]) {
        const int a5 = occ5[s];
        uint32_t hs[3] = {0u, 0u, 0u};
#pragma unroll
        for (int k = 0; k < S; ++k) {
#pragma unroll
            for (int i = 0; i < T; ++i)
                if (a5 == 5 * i) acc[i][k] += h[k];
            if (hist) hs[k] = pack_hist5<T>(h[k], c.pad[k]);
        }
        if (hist) hist[s] = make_uint4(hs[0], hs[1], hs[2], (uint32_t)a5);
        if (++since == 32) {
            flush();
            since = 0;
        }
    };
    if (c.lat.L) {  // implicit neighbours (no sentinel padding: pad[k] == 0)
        lattice_sites<S, uint64_t>(c.lat, threadIdx.x, blockDim.x,
                                   [occ5](int n) { return 1ull << (2 * occ5[n]); }, site);
    } else {
        for (int s = threadIdx.x; s < c.num_sites; s += blockDim.x) {
            uint64_t h[S];
#pragma unroll
            for (int k = 0; k < S; ++k) {
                h[k] = 0;
                const int4 *seg = nbor + (size_t)s * c.row4 + c.off4[k];
                for (int ch = 0; ch < c.chunks[k]; ++ch) {
                    const int4 x = __ldg(seg + ch);
                    h[k] += (1ull << (2 * occ5[x.x])) + (1ull << (2 * occ5[x.y])) + (1ull << (2 * occ5[x.z])) +
                            (1ull << (2 * occ5[x.w]));
                }
            }
            site(s, h);
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
// Random occupancy of population position `pos` of generation `generation`:
// the sorted species layout read through a keyed Feistel permutation (cycle
// walking).  Writes 5*species into occ5 and, when gocc != nullptr, species
// into the slot's row in HBM.  Block-cooperative; no barrier inside.
// ---------------------------------------------------------------------------
template <int T>
__device__ __forceinline__ void generate_occupancy(const SearchConst &c, uint32_t pos, uint32_t generation,
                                                   uint8_t *occ5, uint8_t *gocc)
{
    uint32_t rk[kFeistelRounds];
    const u32x4 w0 = philox4x32_10(u32x4{pos, generation, 0u, kInitStream}, c.key0, c.key1);
    const u32x4 w1 = philox4x32_10(u32x4{pos, generation, 1u, kInitStream}, c.key0, c.key1);
    rk[0] = w0.x; rk[1] = w0.y; rk[2] = w0.z; rk[3] = w0.w; rk[4] = w1.x; rk[5] = w1.y;
    const int n = c.num_sites;
    for (int s = threadIdx.x; s < n; s += blockDim.x) {
        uint32_t y = feistel((uint32_t)s, c.feistel_h, rk);
        while (y >= (uint32_t)n) y = feistel(y, c.feistel_h, rk);
        int t = 0;
#pragma unroll
        for (int i = 1; i < T; ++i) t += (int)(y >= (uint32_t)c.prefix[i]);
        occ5[s] = (uint8_t)(5 * t);
        if (gocc) gocc[s] = (uint8_t)t;
    }
}

// New random occupancy or a recount of a stored one; writes occupancy, counts
// and f2 of the slot.  One CTA per slot; dynamic shared memory = occ_stride +
// 16 + 4*S*T*T bytes.
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
        generate_occupancy<T>(c, blockIdx.x, g.generation, occ5, gocc);
    } else {
        for (int s = threadIdx.x; s < n; s += blockDim.x) occ5[s] = (uint8_t)(5 * gocc[s]);
    }
    if (threadIdx.x == 0) occ5[n] = 0;
    __syncthreads();
    block_recount<T, S>(c, g.nbor, occ5, cnt, g.hist ? g.hist + (size_t)slot * n : nullptr);
    int32_t *gc = g.cnt + (size_t)slot * S * T * T;
    for (int x = threadIdx.x; x < S * T * T; x += blockDim.x) gc[x] = cnt[x];
    if (threadIdx.x == 0) g.f2[slot] = fitness_of_counts<T, S>(c, cnt);
}

// ---------------------------------------------------------------------------
// The local parallel search (pyhea/cpp/accelerate.cpp:601-694): one CTA per
// solution, one lane per task (lanes loop when tasks > blockDim).  Each round
// every task scores one proposal against the same state (its delta D, see
// score_delta); the block takes the (D, task) minimum and accepts it iff
// D < 0; the search ends after `depth` rounds in a row without an accept.
//
// One block barrier per round: each warp publishes its best proposal (a
// SwapRecord, double-buffered by round parity) before the barrier; after it
// every warp reduces the records itself and writes the winning swap into the
// occupancy (all threads write the same two bytes).  On an accept the block
// writes the counts after the swap into the other count buffer, rebuilds the
// table's L half from them and updates the site histograms; a second barrier
// publishes all three before the next round.
//
// Shared memory after the occupancy: the delta table, the records, two count
// buffers (search_smem_tail).
// ---------------------------------------------------------------------------
struct SwapRecord {
    uint64_t key;           // delta_key of the proposal's D
    int32_t task;
    uint32_t s1, s2;
    int32_t ab;             // species a | b << 8 before the swap
    uint32_t h1[3], h2[3];  // shell histograms of both sites, m folded in (score_delta)
    int32_t stop;           // record 0 of a round: the block stops after it (deadline)
    int32_t pad_;
};
static_assert(sizeof(SwapRecord) == 56, "SwapRecord layout");

__host__ __device__ constexpr int mc_ncount_pad(int ncount) { return (ncount + 3) & ~3; }

// Shared-memory bytes of a search after its occupancy: delta table, 2 * nwarps
// swap records, two count buffers.
__host__ __device__ constexpr size_t search_smem_tail(int T, int S, int nwarps)
{
    return (size_t)16 * delta_entries(T, S) + (size_t)2 * nwarps * sizeof(SwapRecord) +
           (size_t)2 * 4 * mc_ncount_pad(S * T * T);
}

struct McTrace {
    AcceptRecord *records;  // trace_cap records for this search, or nullptr
    int32_t *counts;        // trace_cap count snapshots, or nullptr
    int64_t cap;
};

struct McTally {
    double f2;                       // recomputed from the counts, or the running f2 when yielded
    int64_t rounds, accepts, evals;  // rounds run by this call
    int64_t round_end;               // round index the search continues from
    int miss;                        // consecutive rejections at round_end
    int buf;                         // count buffer holding the final counts
    bool yielded;                    // stopped at the deadline before converging
};

// Where a search segment starts: a search stopped at a round boundary
// continues from (round0, miss0) with the same occupancy, counts and running
// f2 and draws the same proposals as one that never stopped.
struct McResume {
    int64_t round0;
    int miss0;
    unsigned long long deadline_ns;  // kYield: stop after the first round ending past this device time (0: never)
    double tol2;                     // kYield: the search ends once its running f2 <= tol2 (< 0: never)
};

// Count change dC_ij of shell k for the accepted swap in record w (a -> b at
// s1, b -> a at s2): sa_i u_j + sa_j u_i with u from the record's histograms.
template <int T>
__device__ __forceinline__ int count_change(const SwapRecord &w, int a, int b, int k, int i, int j)
{
    const uint32_t h1 = w.h1[k], h2 = w.h2[k];
    const int ui = field5(h2, 5 * i) - field5(h1, 5 * i), uj = field5(h2, 5 * j) - field5(h1, 5 * j);
    return ((i == a) - (i == b)) * uj + ((j == a) - (j == b)) * ui;
}

// Delta table of a search starting from the counts in buffer 0 of cnt2
// (the two halves of each entry are written by different threads, so one
// barrier at the end covers both).  Block-wide.
template <int T, int S>
__device__ __forceinline__ void search_setup(const SearchConst &c, const int32_t *cnt2, double2 *tab)
{
    delta_consts<T, S>(c, tab);
    delta_linear<T, S>(c, tab, [cnt2](int k, int i, int j) { return cnt2[(k * T + i) * T + j]; });
    __syncthreads();
}

// Rounds of the local search on the staged state: occupancy occ5, counts in
// buffer 0 of cnt2, the delta table tab (search_setup), running f2 `cur`.
// Every thread returns the same tally; evals is this thread's count.  No
// barrier at entry.  occ5 may be shared or global memory; every thread writes
// the accepted swap's bytes itself, so its own later loads see them either
// way.  The draws read the species from occ5; proposals are scored from the
// site histograms `hist`, which an accept updates.
template <int T, class L, bool kYield = false>
__device__ __forceinline__ McTally mc_rounds(const SearchConst &c, const int4 *__restrict__ nbor, uint8_t *occ5,
                                             int32_t *cnt2, double2 *tab, SwapRecord *rec, uint32_t stream,
                                             double cur, int tasks, int depth, int64_t max_rounds, McTrace tr,
                                             McResume rs, uint4 *hist, const uint32_t *nbmask)
{
    constexpr int S = L::S, NC = S * T * T, NCP = mc_ncount_pad(NC);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    int miss = rs.miss0, buf = 0;
    int64_t round = rs.round0, accepts = 0, evals = 0;
    bool yielded = false;
    while (miss < depth && round < max_rounds && !(kYield && cur <= rs.tol2)) {
        SwapRecord *rr = rec + (round & 1) * nwarps;
        SwapRecord &mine = rr[warp];  // this warp's best proposal of the round
        if (lane == 0) {
            mine.key = kNoSwap;
            mine.task = 0x7FFFFFFF;
        }
        __syncwarp();
        // passes of blockDim tasks; lane q of a pass scores task q (warp-uniform trip count)
        for (int q0 = warp * 32; q0 < tasks; q0 += blockDim.x) {
            const int q = q0 + lane;
            uint32_t s1 = 0, s2 = 0;
            const bool ok = q < tasks && draw_pair(c, stream, (uint32_t)round, (uint32_t)q, occ5, s1, s2);
            __syncwarp();  // lanes that needed more draws rejoin before scoring
            uint64_t key = kNoSwap;
            uint32_t h1[S], h2[S];
            int a = 0, b = 0;
            if (ok) {
                ++evals;
                a = occ5[s1] / 5;
                b = occ5[s2] / 5;
                key = delta_key(score_delta<T, L>(c, nbor, nbmask, tab, load_hist(c, hist + s1), load_hist(c, hist + s2), s1, s2,
                                                  a, b, h1, h2));
            }
            uint64_t wk = key;
            int wq = key != kNoSwap ? q : 0x7FFFFFFF;
            warp_argmin(wk, wq);
            // the lane holding the pass minimum folds it into the warp's record
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
        // the stop decision travels in warp 0's record (read by all after the barrier)
        if (kYield && tid == 0) rr[0].stop = (rs.deadline_ns && global_ns() >= rs.deadline_ns) ? 1 : 0;
        __syncthreads();
        const bool stop = kYield && rr[0].stop != 0;
        // every warp reduces the records of all warps
        uint64_t xk = lane < nwarps ? rr[lane].key : kNoSwap;
        int xq = lane < nwarps ? rr[lane].task : 0x7FFFFFFF;
        const uint64_t own_k = xk;
        const int own_q = xq;
        warp_argmin(xk, xq);
        if (xk != kNoSwap) {
            // the record holding the minimum (tasks of records are distinct)
            const int xw = __ffs(__ballot_sync(0xFFFFFFFFu, own_k == xk && own_q == xq)) - 1;
            const SwapRecord &w = rr[xw];
            const int a = w.ab & 0xFF, b = (w.ab >> 8) & 0xFF;
            occ5[w.s1] = (uint8_t)(5 * b);  // same bytes from every thread
            occ5[w.s2] = (uint8_t)(5 * a);
            const int32_t *cold = cnt2 + buf * NCP;
            int32_t *cnew = cnt2 + (buf ^ 1) * NCP;
            const auto after = [cold, &w, a, b](int k, int i, int j) {
                return cold[(k * T + i) * T + j] + count_change<T>(w, a, b, k, i, j);
            };
            const int me = block_rotation(32 * accept_linear_warps<T, S>());
            for (int x = me; x < NC; x += blockDim.x) cnew[x] = after(x / (T * T), (x / T) % T, x % T);
            delta_linear<T, S>(c, tab, after);
            update_hist<L, false>(c, nbor, hist, w.s1, w.s2, a, b,
                                  block_rotation(32 * (accept_linear_warps<T, S>() + (NC + 31) / 32)));
            const double D = key_delta(xk);
            __syncthreads();  // next round's proposals read the new table and histograms
            buf ^= 1;
            cur = __dadd_rn(cur, D);
            if (tr.records && warp == 0 && accepts < tr.cap) {
                if (lane == 0) {
                    AcceptRecord r;
                    r.round = (uint32_t)round;
                    r.task = (uint32_t)xq;
                    r.s1 = rr[xw].s1;
                    r.s2 = rr[xw].s2;
                    r.f2 = cur;
                    tr.records[accepts] = r;
                }
                if (tr.counts) {
                    int32_t *dst = tr.counts + accepts * NC;
                    for (int x = lane; x < NC; x += 32) dst[x] = cnew[x];
                }
            }
            miss = 0;
            ++accepts;
        } else {
            ++miss;
        }
        ++round;
        if (kYield && stop && miss < depth && round < max_rounds && !(cur <= rs.tol2)) {
            yielded = true;
            break;
        }
    }
    __syncthreads();
    const double f2 = yielded ? cur : fitness_of_counts<T, S>(c, cnt2 + buf * NCP);
    return McTally{f2, round - rs.round0, accepts, evals, round, miss, buf, yielded};
}

// Slot row (species bytes) -> 5*species in shared memory (16-byte vectors).
// kFromL2: load through L2 only (rows written earlier by other CTAs of the
// same launch may sit stale in this SM's L1).
template <bool kFromL2 = false>
__device__ __forceinline__ void stage_occupancy(const SearchConst &c, const uint8_t *gocc, uint8_t *occ5)
{
    const uint4 *src = reinterpret_cast<const uint4 *>(gocc);
    uint4 *dst = reinterpret_cast<uint4 *>(occ5);
    for (int v = threadIdx.x; v < c.occ_stride / 16; v += blockDim.x) {
        uint4 x = kFromL2 ? __ldcg(src + v) : src[v];
        // bytes are species < 8: 5*t per byte without carries
        x.x = x.x * 5u; x.y = x.y * 5u; x.z = x.z * 5u; x.w = x.w * 5u;
        dst[v] = x;
    }
}

// 5*species in shared memory -> slot row (species bytes).
__device__ __forceinline__ void unstage_occupancy(const SearchConst &c, const uint8_t *occ5, uint8_t *gocc)
{
    const uint4 *src = reinterpret_cast<const uint4 *>(occ5);
    uint4 *dst = reinterpret_cast<uint4 *>(gocc);
    for (int v = threadIdx.x; v < c.occ_stride / 16; v += blockDim.x) {
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
}

// Sum of per-thread evaluation counts of the block, added to stats[1];
// rounds and accepts (uniform) to stats[0] and stats[2] by thread 0.
__device__ __forceinline__ void add_tally(const McTally &t, unsigned long long *stats)
{
    unsigned long long ev = (unsigned long long)t.evals;
#pragma unroll
    for (int o = 16; o; o >>= 1) ev += __shfl_xor_sync(0xFFFFFFFFu, ev, o);
    if ((threadIdx.x & 31) == 0 && ev) atomicAdd(&stats[1], ev);
    if (threadIdx.x == 0) {
        atomicAdd(&stats[0], (unsigned long long)t.rounds);
        atomicAdd(&stats[2], (unsigned long long)t.accepts);
    }
}

#ifndef HEA_MC_MIN_BLOCKS
#define HEA_MC_MIN_BLOCKS 2  // resident 512-thread blocks per SM the register budget aims for
#endif
// Shared memory: occ_stride + 16 + search_smem_tail(T, S, nwarps).
template <int T, class L>
__global__ void __launch_bounds__(512, HEA_MC_MIN_BLOCKS) mc_kernel(const SearchConst c, const McArgs g)
{
    constexpr int S = L::S, NC = S * T * T, NCP = mc_ncount_pad(NC);
    extern __shared__ __align__(16) uint8_t smem[];
    const int tid = threadIdx.x, nwarps = blockDim.x >> 5;
    uint8_t *occ5 = smem;
    double2 *tab = reinterpret_cast<double2 *>(smem + c.occ_stride + 16);
    SwapRecord *rec = reinterpret_cast<SwapRecord *>(tab + delta_entries(T, S));  // [2][nwarps]
    int32_t *cnt2 = reinterpret_cast<int32_t *>(rec + 2 * nwarps);                // [2][NCP]

    const int slot = g.order[blockIdx.x];
    const uint32_t stream = (g.mc_call << 16) | (uint32_t)blockIdx.x;
    uint8_t *gocc = g.occ + (size_t)slot * c.occ_stride;
    int32_t *gcnt = g.cnt + (size_t)slot * NC;

    stage_occupancy(c, gocc, occ5);
    for (int x = tid; x < NC; x += blockDim.x) cnt2[x] = gcnt[x];
    __syncthreads();
    if (tid == 0) occ5[c.num_sites] = 0;  // sentinel (occ_stride may end exactly at n)
    search_setup<T, S>(c, cnt2, tab);

    McTrace tr{nullptr, nullptr, 0};
    if (g.trace) {
        tr.records = g.trace + (size_t)blockIdx.x * g.trace_cap;
        tr.counts = g.trace_counts ? g.trace_counts + (size_t)blockIdx.x * g.trace_cap * NC : nullptr;
        tr.cap = g.trace_cap;
    }
    const McTally t = mc_rounds<T, L>(c, g.nbor, occ5, cnt2, tab, rec, stream, g.f2[slot], g.tasks, g.depth,
                                      g.max_rounds, tr, McResume{0, 0, 0ull, -1.0},
                                      g.hist + (size_t)slot * c.num_sites, g.nbmask);

    unstage_occupancy(c, occ5, gocc);
    for (int x = tid; x < NC; x += blockDim.x) gcnt[x] = cnt2[t.buf * NCP + x];
    add_tally(t, g.stats);
    if (tid == 0) {
        g.f2[slot] = t.f2;
        if (g.trace_len) g.trace_len[blockIdx.x] = t.accepts;
        if (g.rounds_out) g.rounds_out[blockIdx.x] = t.rounds;
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
