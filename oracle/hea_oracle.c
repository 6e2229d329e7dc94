/*
 * hea_oracle.c -- CPU restatement of PyHEA's SRO-targeted atom-swap search.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path: only
 * the test suite, the smoke check and the CPU-baseline leg of the benchmark
 * load it.  The product library never links or calls it.
 *
 * What it restates (reference = caimeiniu/pyhea, CPU engine):
 *   - full pair recount          pyhea/cpp/accelerate.cpp:370-399
 *   - fitness of a count matrix  pyhea/cpp/accelerate.cpp:555-569 (and :165-178)
 *   - incremental swap update    pyhea/cpp/accelerate.cpp:512-553
 *   - pair proposal              pyhea/cpp/accelerate.cpp:649-655
 *   - best-of-tasks / accept     pyhea/cpp/accelerate.cpp:643-690
 *   - merge of two populations   pyhea/cpp/accelerate.cpp:305-330
 *   - global loop                pyhea/cpp/accelerate.cpp:713-763
 *
 * The reference draws from std::random_device / std::rand and accumulates the
 * pair fractions as floating-point increments, so no trajectory of it can be
 * replayed.  This restatement fixes every free choice so that a CUDA
 * implementation can be checked bit for bit:
 *
 *   RNG        Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), key = 64-bit
 *              seed.  Proposal counter = {call, task, round, stream},
 *              stream = (mc_call << 16) | slot, two attempts per call.  Bounded draws use Lemire's
 *              multiply-and-reject method (ACM TOMACS 2019), so site draws are
 *              exactly uniform.
 *   Shuffle    a keyed 6-round Feistel permutation with cycle walking (the
 *              same construction family thrust::shuffle uses in the reference
 *              GPU engine, pyhea/cpp/accelerate.cu:925-929); round function is
 *              the murmur3 finaliser; round keys from Philox counter
 *              {slot, generation, 0|1, 0xFFFFFFFF}.
 *   Counts     int32 C[k][i][j] = #{(s, n in shell k of s): occ[s]=i, occ[n]=j};
 *              the reference's gamma is C / (Z_k * N).
 *   Fitness    f2 = sum_k w_k * sum_i sum_j d^2 with d = fma(-C', R, E),
 *              E = 1 - target, R = N / (Z_k * n_i * n_j), accumulated with
 *              fma per shell over the upper triangle row by row (d_ii, then
 *              d_ij, d_ji for j > i).  Fitness reported = sqrt(f2).
 *   Scoring    a proposal is scored by D, the change of f2 its swap makes,
 *              from the rank-2 form of the count change (hea_oracle_delta
 *              below): the same quantity as the reference's full fitness of
 *              the swapped counts (accelerate.cpp:555-569) minus the current
 *              one, in O(T) terms per shell, with a fixed operation order.
 *   Ties       the round's best proposal is the lowest D, lowest task index
 *              on ties; it is accepted iff D < 0 (the reference accepts iff
 *              the new fitness is strictly below the current one,
 *              accelerate.cpp:678); the search's running f2 adds D, and the
 *              f2 stored at its end is recomputed from the counts.
 *              Populations are sorted stably by f2.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define HEA_ORACLE_FEISTEL_ROUNDS 6

/* ------------------------------------------------------------------------ */
/* Philox4x32-10                                                             */
/* ------------------------------------------------------------------------ */
void hea_oracle_philox(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4])
{
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        if (r) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Lemire: accept x iff low32(x*n) >= (2^32 - n) mod n; value = high32(x*n). */
static int bounded(uint32_t x, uint32_t n, uint32_t thresh, uint32_t *v)
{
    uint64_t m = (uint64_t)x * n;
    if ((uint32_t)m < thresh) return 0;
    *v = (uint32_t)(m >> 32);
    return 1;
}

uint32_t hea_oracle_reject_threshold(uint32_t n) { return (uint32_t)(0u - n) % n; }

/* The same on a 16-bit word h (n <= 2^16): accept iff low16(h n) >= 2^16 mod n. */
static int bounded16(uint32_t h, uint32_t n, uint32_t thresh, uint32_t *v)
{
    uint32_t m = h * n;
    if ((m & 0xFFFFu) < thresh) return 0;
    *v = m >> 16;
    return 1;
}

/* 16-bit draws when n <= 2^16 and at most 1/16 of the 16-bit words are rejected. */
int hea_oracle_use_draw16(uint32_t n) { return n <= 65536u && (65536u % n) <= 4096u; }

/*
 * Draw the swap pair for (task, round) of one search stream.  Mirrors the
 * redraw loop at accelerate.cpp:649-655: both sites are redrawn until their
 * species differ.  Philox call c (counter {c, task, round, stream}) carries
 * two attempts, (x0, x1) and then (x2, x3); an attempt is valid when both
 * bounded draws accept and the two species differ.  Returns the index of the
 * attempt used (2c or 2c+1), or -1 when HEA_ORACLE_MAX_CALLS calls found none.
 * With 16-bit draws (hea_oracle_use_draw16), call c carries four attempts:
 * attempt j takes the low and the high half of word x_j (index 4c + j).
 */
#define HEA_ORACLE_MAX_CALLS (1u << 19)
int64_t hea_oracle_draw_pair(const uint32_t key[2], uint32_t stream, uint32_t round, uint32_t task,
                             const uint8_t *occ, uint32_t n, uint32_t *s1, uint32_t *s2)
{
    uint32_t th = hea_oracle_reject_threshold(n);
    if (hea_oracle_use_draw16(n)) {
        uint32_t th16 = 65536u % n;
        for (uint32_t c = 0; c < HEA_ORACLE_MAX_CALLS; ++c) {
            uint32_t ctr[4] = {c, task, round, stream}, x[4];
            hea_oracle_philox(ctr, key, x);
            for (int j = 0; j < 4; ++j) {
                uint32_t u, v;
                if (bounded16(x[j] & 0xFFFFu, n, th16, &u) && bounded16(x[j] >> 16, n, th16, &v) && occ[u] != occ[v]) {
                    *s1 = u;
                    *s2 = v;
                    return (int64_t)(4 * c + j);
                }
            }
        }
        return -1;
    }
    for (uint32_t c = 0; c < HEA_ORACLE_MAX_CALLS; ++c) {
        uint32_t ctr[4] = {c, task, round, stream}, x[4];
        hea_oracle_philox(ctr, key, x);
        for (int half = 0; half < 2; ++half) {
            uint32_t u, v;
            if (bounded(x[2 * half], n, th, &u) && bounded(x[2 * half + 1], n, th, &v) && occ[u] != occ[v]) {
                *s1 = u;
                *s2 = v;
                return (int64_t)(2 * c + half);
            }
        }
    }
    return -1;
}

/* ------------------------------------------------------------------------ */
/* Random occupancy: keyed Feistel permutation of the sorted species layout  */
/* ------------------------------------------------------------------------ */
static uint32_t fmix32(uint32_t h)
{
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}

static int half_bits(uint32_t n)
{
    int b = 0;
    if (n > 1) {
        uint32_t m = n - 1;
        while (m) { ++b; m >>= 1; }
    }
    if (b < 2) b = 2;
    return (b + 1) / 2;
}

static uint32_t feistel(uint32_t x, int h, const uint32_t rk[HEA_ORACLE_FEISTEL_ROUNDS])
{
    uint32_t mask = (h >= 32) ? 0xFFFFFFFFu : ((1u << h) - 1u);
    uint32_t l = x >> h, r = x & mask;
    for (int i = 0; i < HEA_ORACLE_FEISTEL_ROUNDS; ++i) {
        uint32_t nl = r;
        r = l ^ (fmix32(r ^ rk[i]) & mask);
        l = nl;
    }
    return (l << h) | r;
}

void hea_oracle_round_keys(const uint32_t key[2], uint32_t generation, uint32_t slot,
                           uint32_t rk[HEA_ORACLE_FEISTEL_ROUNDS])
{
    uint32_t c0[4] = {slot, generation, 0u, 0xFFFFFFFFu}, c1[4] = {slot, generation, 1u, 0xFFFFFFFFu};
    uint32_t w0[4], w1[4];
    hea_oracle_philox(c0, key, w0);
    hea_oracle_philox(c1, key, w1);
    rk[0] = w0[0]; rk[1] = w0[1]; rk[2] = w0[2]; rk[3] = w0[3]; rk[4] = w1[0]; rk[5] = w1[1];
}

/* Permutation index of site s: cycle-walk the Feistel map until it lands in [0, n). */
uint32_t hea_oracle_permute(uint32_t s, uint32_t n, const uint32_t rk[HEA_ORACLE_FEISTEL_ROUNDS])
{
    int h = half_bits(n);
    uint32_t y = feistel(s, h, rk);
    while (y >= n) y = feistel(y, h, rk);
    return y;
}

/*
 * One random occupancy: the species layout sorted by type (type t repeated
 * species[t] times, accelerate.cpp:236-238) read through the permutation.
 */
void hea_oracle_generate(const uint32_t key[2], uint32_t generation, uint32_t slot, const int32_t *species,
                         int num_types, int num_sites, uint8_t *occ)
{
    uint32_t rk[HEA_ORACLE_FEISTEL_ROUNDS];
    hea_oracle_round_keys(key, generation, slot, rk);
    for (int s = 0; s < num_sites; ++s) {
        uint32_t p = hea_oracle_permute((uint32_t)s, (uint32_t)num_sites, rk);
        int t = 0;
        int64_t acc = species[0];
        while ((int64_t)p >= acc && t + 1 < num_types) acc += species[++t];
        occ[s] = (uint8_t)t;
    }
}

/* ------------------------------------------------------------------------ */
/* Counts, tables, fitness                                                    */
/* ------------------------------------------------------------------------ */
/*
 * Problem description shared by the functions below.  nbor is the flattened
 * neighbour list: row s holds sum(Z) ids, shell 0 first, each shell's ids in
 * the order of the input list (pyhea/lattice/lattice.py:236,256 sorts them).
 */
typedef struct {
    int32_t num_sites, num_types, num_shells, row;
    const int32_t *nbor;
    const int32_t *shell_size;  /* [S]  */
    const int32_t *species;     /* [T]  */
    const double *weight;       /* [S]  */
    const double *E;            /* [S][T][T] = 1 - target */
    const double *R;            /* [S][T][T] = N / (Z_k n_i n_j) */
} hea_oracle_problem;

void hea_oracle_tables(int num_sites, int num_types, int num_shells, const int32_t *shell_size,
                       const int32_t *species, const double *target, double *E, double *R)
{
    int T = num_types;
    for (int k = 0; k < num_shells; ++k)
        for (int i = 0; i < T; ++i)
            for (int j = 0; j < T; ++j) {
                int e = (k * T + i) * T + j;
                E[e] = 1.0 - target[k * T * T + i * T + j];
                R[e] = (double)num_sites / (((double)shell_size[k] * (double)species[i]) * (double)species[j]);
            }
}

void hea_oracle_recount(const hea_oracle_problem *p, const uint8_t *occ, int32_t *C)
{
    int T = p->num_types, S = p->num_shells;
    memset(C, 0, sizeof(int32_t) * (size_t)S * T * T);
    for (int s = 0; s < p->num_sites; ++s) {
        const int32_t *row = p->nbor + (size_t)s * p->row;
        int off = 0;
        for (int k = 0; k < S; ++k) {
            for (int q = 0; q < p->shell_size[k]; ++q) C[(k * T + occ[s]) * T + occ[row[off + q]]] += 1;
            off += p->shell_size[k];
        }
    }
}

/*
 * f2 of a count matrix.  Per shell the squares are accumulated with fma over
 * the upper triangle row by row: the diagonal term d_ii, then for every j > i
 * the pair d_ij, d_ji.  f2 = fma(w_k, e_k, f2) over the shells in order.
 */
static double term_d(const hea_oracle_problem *p, const int32_t *C, int x)
{
    return fma(-(double)C[x], p->R[x], p->E[x]);
}

double hea_oracle_f2(const hea_oracle_problem *p, const int32_t *C)
{
    int T = p->num_types;
    double f2 = 0.0;
    for (int k = 0; k < p->num_shells; ++k) {
        double e = 0.0;
        for (int i = 0; i < T; ++i) {
            double dii = term_d(p, C, (k * T + i) * T + i);
            e = fma(dii, dii, e);
            for (int j = i + 1; j < T; ++j) {
                double dij = term_d(p, C, (k * T + i) * T + j);
                double dji = term_d(p, C, (k * T + j) * T + i);
                e = fma(dij, dij, e);
                e = fma(dji, dji, e);
            }
        }
        f2 = fma(p->weight[k], e, f2);
    }
    return f2;
}

/*
 * Counts after swapping the species of s1 and s2, by the reference's
 * per-neighbour update (accelerate.cpp:512-550): for every neighbour of each
 * swapped site, remove the old ordered pair in both directions and add the new
 * one.  Cp must hold a copy of the current counts on entry.
 */
void hea_oracle_swap_counts(const hea_oracle_problem *p, const uint8_t *occ, uint32_t s1, uint32_t s2, int32_t *Cp)
{
    int T = p->num_types;
    int off = 0;
    for (int k = 0; k < p->num_shells; ++k) {
        int z = p->shell_size[k];
        for (int side = 0; side < 2; ++side) {
            uint32_t c = side ? s2 : s1, o = side ? s1 : s2;
            int atom = occ[c], after = occ[o];
            const int32_t *row = p->nbor + (size_t)c * p->row + off;
            for (int q = 0; q < z; ++q) {
                uint32_t n = (uint32_t)row[q];
                int t = occ[n];
                int tp = (n == o) ? occ[c] : (n == c) ? occ[o] : t;
                Cp[(k * T + atom) * T + t] -= 1;
                Cp[(k * T + t) * T + atom] -= 1;
                Cp[(k * T + after) * T + tp] += 1;
                Cp[(k * T + tp) * T + after] += 1;
            }
        }
        off += z;
    }
}

/* ------------------------------------------------------------------------ */
/* Swap delta                                                                 */
/* ------------------------------------------------------------------------ */
/*
 * Swapping species a (site s1) and b (site s2) changes the counts of shell k
 * only in rows and columns a and b: dC_ij = sa_i u_j + sa_j u_i with
 * sa = e_a - e_b, so that u_t = dC_at for t != a, b, u_a = dC_aa / 2 and
 * u_b = -dC_bb / 2.  Expanding sum_ij (d_ij - R_ij dC_ij)^2 - d_ij^2 with
 * d = E - R C and R symmetric gives, per shell,
 *     sum_t u_t (L_t + u_t Q_t) + (u_a - u_b)^2 Cq
 * with L_t = -2 (G_at - G_bt), G_it = R_it (d_it + d_ti),
 * Q_t = 2 (R_at^2 + R_bt^2) (t != a, b), Q_a = 4 R_aa^2, Q_b = 4 R_bb^2,
 * Cq = 2 R_ab^2; the weights w_k multiply L, Q and Cq.  The tables below hold
 * them for every shell and ordered pair (a, b); L is rebuilt from the counts
 * after every accepted swap.  Operation order (shared with the kernels):
 *     Q = w * (2 * (R_at*R_at + R_bt*R_bt)),  Q_a = w * (4 * (R_aa*R_aa)),
 *     Cq = w * (2 * (R_ab*R_ab)),
 *     d_it = fma(-C_it, R_it, E_it), d_ti = fma(-C_it, R_it, E_ti),
 *     G_it = R_it * (d_it + d_ti),  L = (-2 * w) * (G_at - G_bt),
 *     D = 0; per shell, per t: D = fma(u_t, fma(u_t, Q_t, L_t), D);
 *     then D = fma((u_a - u_b)^2, Cq, D).
 */
typedef struct {
    int T, S;
    double *L;  /* [S][T][T][T]  (k, a, b, t) */
    double *Q;  /* [S][T][T][T] */
    double *Cq; /* [S][T][T] */
} delta_tables;

static int delta_alloc(const hea_oracle_problem *p, delta_tables *d)
{
    size_t n3 = (size_t)p->num_shells * p->num_types * p->num_types * p->num_types;
    d->T = p->num_types;
    d->S = p->num_shells;
    d->L = (double *)calloc(n3, sizeof(double));
    d->Q = (double *)calloc(n3, sizeof(double));
    d->Cq = (double *)calloc((size_t)p->num_shells * p->num_types * p->num_types, sizeof(double));
    return d->L && d->Q && d->Cq;
}

static void delta_free(delta_tables *d)
{
    free(d->L);
    free(d->Q);
    free(d->Cq);
}

static void delta_constants(const hea_oracle_problem *p, delta_tables *d)
{
    int T = d->T;
    for (int k = 0; k < d->S; ++k) {
        const double *R = p->R + (size_t)k * T * T;
        double w = p->weight[k];
        for (int a = 0; a < T; ++a)
            for (int b = 0; b < T; ++b) {
                if (a == b) continue;
                size_t row = ((size_t)(k * T + a) * T + b);
                d->Cq[row] = w * (2.0 * (R[a * T + b] * R[a * T + b]));
                for (int t = 0; t < T; ++t) {
                    double q;
                    if (t == a || t == b)
                        q = w * (4.0 * (R[t * T + t] * R[t * T + t]));
                    else
                        q = w * (2.0 * (R[a * T + t] * R[a * T + t] + R[b * T + t] * R[b * T + t]));
                    d->Q[row * T + t] = q;
                }
            }
    }
}

static void delta_linear(const hea_oracle_problem *p, const int32_t *C, delta_tables *d)
{
    int T = d->T;
    double *G = (double *)malloc(sizeof(double) * (size_t)T * T);
    for (int k = 0; k < d->S; ++k) {
        const double *R = p->R + (size_t)k * T * T, *E = p->E + (size_t)k * T * T;
        const int32_t *Ck = C + (size_t)k * T * T;
        for (int i = 0; i < T; ++i)
            for (int t = 0; t < T; ++t) {
                double c = (double)Ck[i * T + t];
                double dit = fma(-c, R[i * T + t], E[i * T + t]);
                double dti = fma(-c, R[i * T + t], E[t * T + i]);
                G[i * T + t] = R[i * T + t] * (dit + dti);
            }
        double m2w = -2.0 * p->weight[k];
        for (int a = 0; a < T; ++a)
            for (int b = 0; b < T; ++b) {
                if (a == b) continue;
                for (int t = 0; t < T; ++t)
                    d->L[((size_t)(k * T + a) * T + b) * T + t] = m2w * (G[a * T + t] - G[b * T + t]);
            }
    }
    free(G);
}

/* D of the swap whose counts before and after are C and Cp (a at s1, b at s2). */
static double delta_of(const delta_tables *d, const int32_t *C, const int32_t *Cp, int a, int b)
{
    int T = d->T;
    double D = 0.0;
    for (int k = 0; k < d->S; ++k) {
        const int32_t *c0 = C + (size_t)k * T * T, *c1 = Cp + (size_t)k * T * T;
        size_t row = (size_t)(k * T + a) * T + b;
        int ua = 0, ub = 0;
        for (int t = 0; t < T; ++t) {
            int u;
            if (t == a)
                u = (c1[a * T + a] - c0[a * T + a]) / 2;
            else if (t == b)
                u = -(c1[b * T + b] - c0[b * T + b]) / 2;
            else
                u = c1[a * T + t] - c0[a * T + t];
            if (t == a) ua = u;
            if (t == b) ub = u;
            double ud = (double)u;
            D = fma(ud, fma(ud, d->Q[row * T + t], d->L[row * T + t]), D);
        }
        D = fma((double)((ua - ub) * (ua - ub)), d->Cq[row], D);
    }
    return D;
}

/*
 * D of swapping s1 and s2 (species must differ) in the state (occ, C): the
 * tables are built from C, the swapped counts by the reference's update.
 */
double hea_oracle_delta(const hea_oracle_problem *p, const uint8_t *occ, const int32_t *C, uint32_t s1, uint32_t s2)
{
    size_t ncount = (size_t)p->num_shells * p->num_types * p->num_types;
    delta_tables d;
    int32_t *cp = (int32_t *)malloc(sizeof(int32_t) * ncount);
    if (!cp || !delta_alloc(p, &d)) return NAN;
    delta_constants(p, &d);
    delta_linear(p, C, &d);
    memcpy(cp, C, sizeof(int32_t) * ncount);
    hea_oracle_swap_counts(p, occ, s1, s2, cp);
    double D = delta_of(&d, C, cp, occ[s1], occ[s2]);
    delta_free(&d);
    free(cp);
    return D;
}

/* ------------------------------------------------------------------------ */
/* Local parallel Monte Carlo on one solution (accelerate.cpp:626-692)       */
/* ------------------------------------------------------------------------ */
typedef struct {
    uint32_t round, task, s1, s2;
    double f2;
} hea_oracle_accept;

/*
 * Runs the swap search on one occupancy in place.  C holds its counts on entry
 * and on exit; *f2 its fitness on entry and, on exit, the fitness recomputed
 * from the final counts.  Returns the number of rounds; each round scores
 * `tasks` proposals.  When trace != NULL up to trace_cap accepted swaps are
 * written there with the running f2 after each (and, when trace_counts !=
 * NULL, the counts after each of them).
 */
int64_t hea_oracle_mc(const hea_oracle_problem *p, const uint32_t key[2], uint32_t stream, int tasks, int depth,
                      int64_t max_rounds, uint8_t *occ, int32_t *C, double *f2, hea_oracle_accept *trace,
                      int32_t *trace_counts, int64_t trace_cap, int64_t *n_accepts, int64_t *n_evals)
{
    size_t ncount = (size_t)p->num_shells * p->num_types * p->num_types;
    int32_t *cp = (int32_t *)malloc(sizeof(int32_t) * ncount);
    int32_t *cbest = (int32_t *)malloc(sizeof(int32_t) * ncount);
    delta_tables d;
    if (!cp || !cbest || !delta_alloc(p, &d)) return -1;
    delta_constants(p, &d);
    delta_linear(p, C, &d);
    double cur = *f2;
    int64_t rounds = 0, acc = 0, evals = 0;
    int miss = 0;
    while (miss < depth && rounds < max_rounds) {
        double best = 0.0;
        int64_t bq = -1;
        uint32_t b1 = 0, b2 = 0;
        for (int q = 0; q < tasks; ++q) {
            uint32_t s1, s2;
            if (hea_oracle_draw_pair(key, stream, (uint32_t)rounds, (uint32_t)q, occ, (uint32_t)p->num_sites, &s1, &s2) < 0)
                continue;
            ++evals;
            memcpy(cp, C, sizeof(int32_t) * ncount);
            hea_oracle_swap_counts(p, occ, s1, s2, cp);
            double D = delta_of(&d, C, cp, occ[s1], occ[s2]);
            if (D < 0.0 && (bq < 0 || D < best)) {
                best = D;
                bq = q;
                b1 = s1;
                b2 = s2;
                memcpy(cbest, cp, sizeof(int32_t) * ncount);
            }
        }
        if (bq >= 0) {
            uint8_t t = occ[b1];
            occ[b1] = occ[b2];
            occ[b2] = t;
            memcpy(C, cbest, sizeof(int32_t) * ncount);
            delta_linear(p, C, &d);
            cur = cur + best;
            miss = 0;
            if (trace && acc < trace_cap) {
                trace[acc].round = (uint32_t)rounds;
                trace[acc].task = (uint32_t)bq;
                trace[acc].s1 = b1;
                trace[acc].s2 = b2;
                trace[acc].f2 = cur;
                if (trace_counts) memcpy(trace_counts + (size_t)acc * ncount, C, sizeof(int32_t) * ncount);
            }
            ++acc;
        } else {
            ++miss;
        }
        ++rounds;
    }
    free(cp);
    free(cbest);
    delta_free(&d);
    *f2 = hea_oracle_f2(p, C);
    if (n_accepts) *n_accepts = acc;
    if (n_evals) *n_evals = evals;
    return rounds;
}

/* ------------------------------------------------------------------------ */
/* Global search (accelerate.cpp:713-763)                                     */
/* ------------------------------------------------------------------------ */
/* Stable order of n fitness values: perm[r] = index of the r-th smallest. */
static void stable_order(const double *f, int n, int *perm)
{
    for (int i = 0; i < n; ++i) perm[i] = i;
    /* insertion sort keeps equal keys in index order; n is a population size */
    for (int i = 1; i < n; ++i) {
        int v = perm[i], j = i - 1;
        while (j >= 0 && f[perm[j]] > f[v]) {
            perm[j + 1] = perm[j];
            --j;
        }
        perm[j + 1] = v;
    }
}

static void reorder(uint8_t *occ, double *f2, int n, int num_sites, const int *perm, uint8_t *tmp_occ, double *tmp_f)
{
    for (int r = 0; r < n; ++r) {
        memcpy(tmp_occ + (size_t)r * num_sites, occ + (size_t)perm[r] * num_sites, (size_t)num_sites);
        tmp_f[r] = f2[perm[r]];
    }
    memcpy(occ, tmp_occ, (size_t)n * num_sites);
    memcpy(f2, tmp_f, sizeof(double) * (size_t)n);
}

typedef struct {
    int64_t rounds, evals, accepts;
} hea_oracle_stats;

/*
 * The whole search: initial population (generation 0), then per iteration a
 * new population (generation it+1) searched with mc_call 2*it, merged with the
 * current one (best P of 2P, stable), and the survivors searched with mc_call
 * 2*it+1.  Output: occupancies [P][N] and f2 [P], ascending after the last
 * iteration.
 */
int hea_oracle_hcs(const hea_oracle_problem *p, const uint32_t key[2], int num_solutions, int total_iter, int tasks,
                   int depth, int64_t max_rounds, uint8_t *out_occ, double *out_f2, hea_oracle_stats *stats)
{
    int P = num_solutions, N = p->num_sites;
    size_t ncount = (size_t)p->num_shells * p->num_types * p->num_types;
    uint8_t *both = (uint8_t *)malloc((size_t)2 * P * N);
    uint8_t *tmp = (uint8_t *)malloc((size_t)2 * P * N);
    double *f = (double *)malloc(sizeof(double) * 2 * P);
    double *tf = (double *)malloc(sizeof(double) * 2 * P);
    int *perm = (int *)malloc(sizeof(int) * 2 * P);
    int32_t *C = (int32_t *)malloc(sizeof(int32_t) * ncount);
    if (!both || !tmp || !f || !tf || !perm || !C) return -1;
    hea_oracle_stats st = {0, 0, 0};

    for (int s = 0; s < P; ++s) {
        hea_oracle_generate(key, 0, (uint32_t)s, p->species, p->num_types, N, both + (size_t)s * N);
        hea_oracle_recount(p, both + (size_t)s * N, C);
        f[s] = hea_oracle_f2(p, C);
    }
    for (int it = 0; it < total_iter; ++it) {
        uint8_t *nw = both + (size_t)P * N;
        for (int half = 0; half < 2; ++half) {
            uint8_t *pop = half ? both : nw;
            double *pf = half ? f : f + P;
            uint32_t call = (uint32_t)(2 * it + half);
            for (int s = 0; s < P; ++s) {
                uint8_t *o = pop + (size_t)s * N;
                if (!half) {
                    hea_oracle_generate(key, (uint32_t)(it + 1), (uint32_t)s, p->species, p->num_types, N, o);
                    hea_oracle_recount(p, o, C);
                    pf[s] = hea_oracle_f2(p, C);
                } else {
                    hea_oracle_recount(p, o, C);
                }
                int64_t acc = 0, ev = 0;
                st.rounds += hea_oracle_mc(p, key, (call << 16) | (uint32_t)s, tasks, depth, max_rounds, o, C, &pf[s],
                                           NULL, NULL, 0, &acc, &ev);
                st.accepts += acc;
                st.evals += ev;
            }
            stable_order(pf, P, perm);
            reorder(pop, pf, P, N, perm, tmp, tf);
            if (!half) {
                /* merge: current population first, then the new one (accelerate.cpp:315-325) */
                stable_order(f, 2 * P, perm);
                reorder(both, f, 2 * P, N, perm, tmp, tf);
            }
        }
    }
    memcpy(out_occ, both, (size_t)P * N);
    memcpy(out_f2, f, sizeof(double) * P);
    if (stats) *stats = st;
    free(both); free(tmp); free(f); free(tf); free(perm); free(C);
    return 0;
}
