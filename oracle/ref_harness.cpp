/*
 * ref_harness.cpp -- C entry points into the reference CPU engine.
 *
 * TEST INFRASTRUCTURE ONLY.  The recipe in oracle/build_oracle.py compiles
 * this file together with the reference's own source
 * (pyhea/cpp/accelerate.cpp, included below from the reference tree, never
 * copied) and the single-rank MPI stub into oracle/_ref/libref_accelerate.so.
 * The tests use it to pin the CPU restatement (hea_oracle.c) against the
 * reference functions, and the benchmark's reference arm times the reference
 * engine through ref_run_local_parallel_hcs.
 *
 * Wrapped reference symbols:
 *   accelerate::cpu::calculate_sro_coefficient     accelerate.cpp:370-399
 *   accelerate::cpu::calculate_fitness_incremental accelerate.cpp:498-570
 *   accelerate::cpu::calculate_fitness_of_solutions accelerate.cpp:118-180
 *   accelerate::cpu::run_local_parallel_hcs        accelerate.cpp:713-763
 * and counts the engine's swap evaluations (below).
 */
#include <dlfcn.h>

#include <cstdint>
#include <cstdlib>
#include <tuple>
#include <vector>

/*
 * Call counter on the C library's rand(), which the reference engine uses for
 * every swap proposal (accelerate.cpp:649-655, two calls per attempt).  The
 * library is linked with -Bsymbolic-functions so the engine's calls bind here;
 * each call is forwarded to the C library's own rand, so the engine's random
 * stream is the stock one.
 */
static unsigned long long g_rand_calls = 0;
extern "C" int rand(void) noexcept
{
    static int (*real_rand)(void) = nullptr;
    if (!real_rand) real_rand = reinterpret_cast<int (*)(void)>(dlsym(RTLD_NEXT, "rand"));
    ++g_rand_calls;
    return real_rand();
}

/*
 * Evaluation counter.  The reference's local search scores every proposal
 * with one call of calculate_fitness_incremental (accelerate.cpp:659-661,
 * an unqualified call on std::vector arguments).  Argument-dependent lookup
 * at that call also finds the non-template function below, declared in the
 * arguments' namespace before the reference source is read; with identical
 * parameter types a non-template is preferred over the template, so each call
 * passes through here, is counted, and runs the reference's own template.
 */
static unsigned long long g_fitness_calls = 0;
namespace accelerate {
namespace cpu {
template <typename Integer, typename Real>
Real calculate_fitness_incremental(std::vector<Integer> &lattice, std::vector<std::vector<std::vector<Real>>> &gamma,
                                   const Integer &atom1, const Integer &atom2, const Integer &num_atoms,
                                   const Integer &num_types, const Integer &num_shells,
                                   const std::vector<Integer> &species,
                                   const std::vector<std::vector<std::vector<Integer>>> &neighbor_list,
                                   const std::vector<std::vector<Real>> &target_sro, const std::vector<Real> &weight);
}  // namespace cpu
}  // namespace accelerate
namespace std {
double calculate_fitness_incremental(vector<int> &lattice, vector<vector<vector<double>>> &gamma, const int &atom1,
                                     const int &atom2, const int &num_atoms, const int &num_types,
                                     const int &num_shells, const vector<int> &species,
                                     const vector<vector<vector<int>>> &neighbor_list,
                                     const vector<vector<double>> &target_sro, const vector<double> &weight)
{
    ++g_fitness_calls;
    return accelerate::cpu::calculate_fitness_incremental<int, double>(lattice, gamma, atom1, atom2, num_atoms,
                                                                       num_types, num_shells, species, neighbor_list,
                                                                       target_sro, weight);
}
}  // namespace std

#include "accelerate.cpp"

using accelerate::cpu::calculate_fitness_incremental;
using accelerate::cpu::calculate_fitness_of_solutions;
using accelerate::cpu::calculate_sro_coefficient;

namespace {
using vec3i = std::vector<std::vector<std::vector<int>>>;
using vec3d = std::vector<std::vector<std::vector<double>>>;

vec3i unflatten_nbor(int num_sites, int num_shells, const int32_t *nbor, int row, const int32_t *shell_size)
{
    vec3i out(num_sites, std::vector<std::vector<int>>(num_shells));
    for (int s = 0; s < num_sites; ++s) {
        int off = 0;
        for (int k = 0; k < num_shells; ++k) {
            out[s][k].assign(nbor + (size_t)s * row + off, nbor + (size_t)s * row + off + shell_size[k]);
            off += shell_size[k];
        }
    }
    return out;
}

std::vector<std::vector<double>> unflatten_target(int num_shells, int num_types, const double *target)
{
    std::vector<std::vector<double>> t(num_shells);
    for (int k = 0; k < num_shells; ++k)
        t[k].assign(target + (size_t)k * num_types * num_types, target + (size_t)(k + 1) * num_types * num_types);
    return t;
}
}  // namespace

extern "C" {

unsigned long long ref_rand_calls(void) { return g_rand_calls; }
void ref_reset_rand_calls(void) { g_rand_calls = 0; }
/* Swap evaluations (calls of the reference's incremental fitness) since the last reset. */
unsigned long long ref_eval_count(void) { return g_fitness_calls; }
void ref_reset_eval_count(void) { g_fitness_calls = 0; }

/* gamma[i][j][k] (reference layout) of one occupancy. */
int ref_recount(int num_sites, int num_types, int num_shells, const int32_t *nbor, int row,
                const int32_t *shell_size, const int32_t *species, const int32_t *occ, double *gamma_out)
{
    vec3i nl = unflatten_nbor(num_sites, num_shells, nbor, row, shell_size);
    std::vector<int> lat(occ, occ + num_sites), sp(species, species + num_types);
    vec3d g(num_types, std::vector<std::vector<double>>(num_types, std::vector<double>(num_shells, 0.0)));
    int n = num_sites, t = num_types, s = num_shells;
    calculate_sro_coefficient<int, double>(g, n, t, s, lat, sp, nl);
    for (int i = 0; i < t; ++i)
        for (int j = 0; j < t; ++j)
            for (int k = 0; k < s; ++k) gamma_out[(i * t + j) * s + k] = g[i][j][k];
    return 0;
}

/*
 * The reference's incremental fitness for swapping (atom1, atom2) of occ,
 * starting from gamma_in (reference layout); writes the updated gamma.
 */
double ref_fitness_incremental(int num_sites, int num_types, int num_shells, const int32_t *nbor, int row,
                               const int32_t *shell_size, const int32_t *species, const double *weight,
                               const double *target, const int32_t *occ, int atom1, int atom2,
                               const double *gamma_in, double *gamma_out)
{
    vec3i nl = unflatten_nbor(num_sites, num_shells, nbor, row, shell_size);
    std::vector<int> lat(occ, occ + num_sites), sp(species, species + num_types);
    std::vector<double> w(weight, weight + num_shells);
    auto tg = unflatten_target(num_shells, num_types, target);
    int n = num_sites, t = num_types, s = num_shells;
    vec3d g(t, std::vector<std::vector<double>>(t, std::vector<double>(s, 0.0)));
    for (int i = 0; i < t; ++i)
        for (int j = 0; j < t; ++j)
            for (int k = 0; k < s; ++k) g[i][j][k] = gamma_in[(i * t + j) * s + k];
    double f = calculate_fitness_incremental<int, double>(lat, g, atom1, atom2, n, t, s, sp, nl, tg, w);
    for (int i = 0; i < t; ++i)
        for (int j = 0; j < t; ++j)
            for (int k = 0; k < s; ++k) gamma_out[(i * t + j) * s + k] = g[i][j][k];
    return f;
}

/* The reference's full-recount fitness of P occupancies [P][N]. */
int ref_fitness_of_solutions(int num_solutions, int num_sites, int num_types, int num_shells, const int32_t *nbor,
                             int row, const int32_t *shell_size, const int32_t *species, const double *weight,
                             const double *target, const int32_t *occ, double *fitness_out)
{
    vec3i nl = unflatten_nbor(num_sites, num_shells, nbor, row, shell_size);
    std::vector<std::vector<int>> lats(num_solutions);
    for (int p = 0; p < num_solutions; ++p) lats[p].assign(occ + (size_t)p * num_sites, occ + (size_t)(p + 1) * num_sites);
    std::vector<int> sp(species, species + num_types);
    std::vector<double> w(weight, weight + num_shells), sro(num_shells, 0.0), fit(num_solutions, 0.0);
    auto tg = unflatten_target(num_shells, num_types, target);
    calculate_fitness_of_solutions<int, double>(fit, lats, sro, w, sp, nl, tg);
    for (int p = 0; p < num_solutions; ++p) fitness_out[p] = fit[p];
    return 0;
}

/* The reference CPU engine end to end (one rank): occ_out [P][N], fitness_out [P]. */
int ref_run_local_parallel_hcs(int num_solutions, int step, int task, int depth, double thr, int num_sites,
                               int num_types, int num_shells, const int32_t *nbor, int row, const int32_t *shell_size,
                               const int32_t *species, const double *weight, const double *target, int32_t *occ_out,
                               double *fitness_out)
{
    vec3i nl = unflatten_nbor(num_sites, num_shells, nbor, row, shell_size);
    std::vector<int> sp(species, species + num_types);
    std::vector<double> w(weight, weight + num_shells);
    auto tg = unflatten_target(num_shells, num_types, target);
    auto res = accelerate::cpu::run_local_parallel_hcs(num_solutions, step, task, depth, thr, nl, sp, w, tg);
    const auto &lats = std::get<0>(res);
    const auto &fit = std::get<1>(res);
    for (size_t p = 0; p < lats.size(); ++p) {
        for (int s = 0; s < num_sites; ++s) occ_out[p * num_sites + s] = lats[p][s];
        fitness_out[p] = fit[p];
    }
    return (int)lats.size();
}

}  // extern "C"
