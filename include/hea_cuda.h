/*
 * hea_cuda.h -- C ABI of the B200 swap-search engine (libhea_cuda.so).
 *
 * The engine replaces the GPU engine of PyHEA, i.e. the function bound by
 * pyhea/cpp/bind.cpp:49-58 as accelerate.run_local_parallel_hcs_cuda and
 * declared at pyhea/cpp/accelerate.h:51-60 (implemented at
 * pyhea/cpp/accelerate.cu:1112-1242).  All pointers here are plain host
 * pointers; the library owns every device buffer it uses.  No call exits the
 * process: each returns HEA_OK or an error code, and hea_last_error() gives the
 * message of the calling thread's last failure.
 *
 * Neighbour table layout (the flattened form of pyhea/lattice/lattice.py:
 * 196-323 output, cut to the first num_shells shells as accelerate.cu:1139-1141
 * does): nbor[s * row + off_k + q] is the q-th neighbour of site s in shell k,
 * row = sum of shell_sizes, off_k = sum of the sizes before k.
 */
#ifndef HEA_CUDA_H
#define HEA_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HEA_OK 0
#define HEA_ERR_INVALID 1     /* an argument is out of range or inconsistent      */
#define HEA_ERR_UNSUPPORTED 2 /* valid input outside what the kernels implement    */
#define HEA_ERR_CUDA 3        /* the CUDA runtime reported an error                */
#define HEA_ERR_NOMEM 4       /* a device or host allocation failed                */

#define HEA_FLAG_LOG_ITERS 1    /* print the per-iteration best fitness line, as accelerate.cu:1208-1212 does */
#define HEA_FLAG_TIME_KERNELS 2 /* time every local-search launch with CUDA events (hea_stats.mc_ms)        */
#define HEA_FLAG_HBM_OCCUPANCY 4 /* keep occupancies in HBM and search each solution with a thread-block
                                    cluster -- the path structures too large for shared memory always take */
#define HEA_FLAG_AUTOTUNE 8     /* plans: time the local search's CTA sizes on short searches at creation
                                   and keep the fastest (results do not depend on it); cached per shape */

/* One structure to search.  Mirrors the arguments nbor, element, weight and
 * target_sro of run_local_parallel_hcs_cuda (bind.cpp:55-58). */
typedef struct hea_problem {
    int32_t num_sites;           /* N = sum of species (accelerate.cu:1128)          */
    int32_t num_types;           /* T = len(element), 2..6                            */
    int32_t num_shells;          /* S = len(weight), 1..3 (accelerate.cu:1126)        */
    const int32_t *shell_sizes;  /* [S] neighbours per site in each shell             */
    const int32_t *nbor;         /* [N][sum shell_sizes] neighbour ids                */
    const int32_t *species;      /* [T] atoms of each species ("element")             */
    const double *weight;        /* [S] shell weights                                 */
    const double *target_sro;    /* [S][T*T] target Warren-Cowley alpha, row-major    */
    /* Optional implicit neighbours (no counterpart in the reference, which
     * always passes a table, lattice.py:196-323): with nbor == NULL, a perfect
     * FCC/BCC cube described here stands for the table, its neighbour ids are
     * computed on the device from lattice arithmetic and no table is stored.
     * implicit_lattice: 1 FCC, 2 BCC; lattice_cell: the cube's edge in unit
     * cells (N = 4 or 2 cell^3); lattice_shell_set as in hea_build_neighbors.
     * shell_sizes must be the lattice's for the first S shells.  Results equal
     * those with the table hea_build_neighbors builds.
     * With a table (nbor != NULL), implicit_lattice 0 lets the library
     * recognise an FCC/BCC cube's table -- every shell of every site holding
     * the ids hea_build_neighbors gives, in any order, as PyHEA's lattice
     * tables do -- and run it on lattice arithmetic instead (same results; the
     * table is not kept); -1 uses the table as given.  Plans report which form
     * they run (hea_plan_lattice). */
    int32_t implicit_lattice;
    int32_t lattice_cell;
    int32_t lattice_shell_set;
} hea_problem;

/* Search controls: nnet, step, task, depth, thr of the reference call
 * (bind.cpp:50-54), plus the seed the reference does not take. */
typedef struct hea_params {
    int32_t num_solutions;  /* nnet: population size P                               */
    int32_t total_iter;     /* step: global iterations I                             */
    int32_t parallel_task;  /* task: proposals scored per round Q                    */
    int32_t converge_depth; /* depth: rounds without improvement that end a search   */
    double threshold;       /* thr: accepted and unused, as in the reference         */
    uint64_t seed;          /* Philox key of every random draw of the search         */
    int64_t max_rounds;     /* cap on rounds per local search (<= 0: 2^31)           */
    int32_t flags;          /* HEA_FLAG_*                                            */
} hea_params;

typedef struct hea_stats {
    int64_t rounds;   /* search rounds over all local searches                      */
    int64_t evals;    /* swap evaluations (proposals scored)                        */
    int64_t accepts;  /* accepted swaps                                             */
    double gpu_ms;    /* device time of the search, CUDA events                     */
    double mc_ms;     /* summed device time of the local-search launches (HEA_FLAG_TIME_KERNELS) */
    int64_t mc_launches; /* local-search launches timed                             */
} hea_stats;

typedef struct hea_accept_record {
    uint32_t round, task, s1, s2;
    double f2;
} hea_accept_record;

/* accelerate::gpu::cuda_available (accelerate.cu:33-37): 1 if a CUDA device is usable. */
int hea_cuda_available(void);

/* Message of the calling thread's last failed call ("" if none). */
const char *hea_last_error(void);

/* Device buffers of finished searches are cached for the next search of the
 * same shape (up to 8 GiB per process); this returns the current device's
 * cached buffers to the driver.  No counterpart in the reference. */
void hea_release_cached_memory(void);

/* L2 read bandwidth of the current device, the denominator of the search
 * kernels' L2 roofline (their tables and site histograms stay in L2 at the
 * benchmark sizes): every SM reads a buffer of `bytes` (it must fit in L2;
 * 16-byte loads through L2 only) `reps` times after one warm-up pass; *out_gbs
 * = bytes * reps / CUDA-event time.  A measurement aid with no counterpart in
 * the reference. */
int hea_l2_read_probe(int64_t bytes, int32_t reps, double *out_gbs);

/* Random 16-byte loads per second from a buffer of `bytes` (far larger than
 * L2), per_thread loads by each thread of 8 and of 32 CTAs x 256 threads per
 * SM, L2-cached and evict-first, each after one warm-up launch; the best rate:
 * the ceiling of the site-histogram loads of structures whose histograms stay
 * in DRAM (each such load brings a 128-byte line from DRAM on B200).  A
 * measurement aid with no counterpart in the reference. */
int hea_dram_random_probe(int64_t bytes, int32_t per_thread, double *out_loads_per_s);

/*
 * The whole search, host buffers in and out: replaces
 * accelerate::gpu::run_local_parallel_hcs_cuda (accelerate.cu:1112-1242).
 * out_occ [P][N] receives species ids, out_fitness [P] the fitness
 * sqrt(f2), both ascending by fitness (the order the reference returns,
 * pyhea/model/opt.py:103-114 writes entry 0).  stats may be NULL.
 */
int hea_run_local_parallel_hcs(const hea_problem *problem, const hea_params *params, uint8_t *out_occ,
                               double *out_fitness, hea_stats *stats);

/*
 * Device-resident form of the same search for repeated runs: create uploads
 * the tables once; run executes the search on the plan's stream and waits for
 * it; read copies the result out.  Same results as hea_run_local_parallel_hcs
 * for the same seed.  There is no counterpart call in the reference; it splits
 * hea_run_local_parallel_hcs at its host/device boundary.
 */
typedef struct hea_plan hea_plan;
int hea_plan_create(const hea_problem *problem, const hea_params *params, hea_plan **out);
int hea_plan_run(hea_plan *plan, uint64_t seed, hea_stats *stats);
int hea_plan_read(hea_plan *plan, uint8_t *out_occ, double *out_fitness);
void hea_plan_destroy(hea_plan *plan);
/* Threads per CTA of the plan's local search (the autotuner's pick with HEA_FLAG_AUTOTUNE). */
int32_t hea_plan_local_search_block(const hea_plan *plan);
/* Neighbours of the plan's structure: 0 from its table, 1 (FCC) or 2 (BCC)
 * from lattice arithmetic (implicit, or a recognised lattice table). */
int32_t hea_plan_lattice(const hea_plan *plan);

/*
 * Batched search: `count` independent structures (each with its own problem,
 * parameters and seed) searched together by one persistent kernel, the run
 * captured once as a CUDA graph.  Each structure's result is identical to
 * hea_run_local_parallel_hcs on that structure alone with the same seed.
 * There is no counterpart in the reference, which searches one structure per
 * call (accelerate.cu:1112-1242); this batches many such calls.
 * run: seeds [count] (NULL keeps the previous ones); read: structure index's
 * occupancies [P][N] and fitness [P], ascending.
 */
typedef struct hea_batch hea_batch;
int hea_batch_create(const hea_problem *problems, const hea_params *params, int32_t count, hea_batch **out);
int hea_batch_run(hea_batch *batch, const uint64_t *seeds, hea_stats *stats);
int hea_batch_read(hea_batch *batch, int32_t index, uint8_t *out_occ, double *out_fitness);
/* Milliseconds from the start of the last run to each structure's final sort (device clock). */
int hea_batch_finish_times(hea_batch *batch, double *out_ms);
/* Per structure of the last run: local-search rounds, swap evaluations and
 * accepted swaps, out[count][3] (the same counts as hea_stats of searching the
 * structure alone with the same seed). */
int hea_batch_tallies(hea_batch *batch, uint64_t *out);
/* Autotuner of the batch's launch: times full runs (with the current seeds) for
 * occupancy kept in HBM or staged in shared memory where it fits, at the
 * kernel's resident CTAs per SM or one fewer, and keeps the fastest.  Results
 * do not depend on the choice.  Outputs may be NULL. */
int hea_batch_autotune(hea_batch *batch, int32_t *out_hbm_all, int32_t *out_ctas_per_sm);
/* Bound on every wait of the persistent kernel for queued work (default 60 s):
 * a CTA that finds no job for this long after the last finished one sets the
 * batch's error flag and every CTA returns; hea_batch_run then fails with a
 * message and the next run starts clean.  No counterpart in the reference
 * (its kernels never wait on one another). */
int hea_batch_set_wait_limit(hea_batch *batch, double ms);
void hea_batch_destroy(hea_batch *batch);

/*
 * Serving loop: structure-search requests admitted while others run.  No
 * counterpart in the reference, whose engine searches one structure per call
 * (accelerate.cu:1112-1242).  Without a tolerance a request's result is
 * identical to hea_run_local_parallel_hcs on it alone with the same seed;
 * with one, to the same request served alone.  Neither depends on what else
 * was on the GPU or where the time slices fell.
 *
 * submit queues a request on the host (inputs are copied); step waits for
 * the previous time slice, hands over the requests that finished in it,
 * admits queued requests in submission order while a request slot, device
 * memory in the arena and job-ring room are free, and launches the persistent
 * search kernel for the next slice (slice_ms, or until nothing is active)
 * without waiting for it -- the host's work between steps overlaps the GPU's;
 * result hands over a finished request's population (ascending fitness) and
 * releases it.  tolerance >= 0 (on the reported fitness, sqrt
 * of f2): a local search ends once its fitness is <= tolerance, and the
 * request ends once the best fitness after an iteration's survivors' sort
 * is; < 0 runs total_iter iterations.  priority 0..15, 0 first.
 * submit_lattice builds the FCC/BCC table on the device (as
 * hea_build_neighbors; the first num_shells shells are searched).
 * result returns HEA_PENDING while the request is queued or running.
 * Not thread-safe: one host thread drives a server.
 */
#define HEA_PENDING 5 /* hea_server_result: the request has not finished */

typedef struct hea_server_config {
    int32_t max_requests;  /* requests on the device at once (0: 256)                            */
    int32_t ring_jobs;     /* job-ring slots per priority level (0: 65536)                        */
    int64_t arena_bytes;   /* device memory for tables and populations (0: 8 GiB or half the free memory) */
    int32_t smem_bytes;    /* shared memory per CTA; larger structures keep occupancy in HBM (0: auto) */
    int32_t hbm_sites;     /* occupancy in HBM for structures of at least this many sites; 0: all (the
                              default, fastest with histogram scoring); -1: only those beyond smem_bytes */
    double slice_ms;       /* length of one step's launch (0: 20 ms)                             */
    double wait_limit_ms;  /* bound on every wait inside the kernel for queued work (0: 10 s); a CTA
                              whose wait runs out stops the slice with an error and the server stops */
} hea_server_config;

typedef struct hea_request_info {
    int32_t state;        /* 0 queued, 1 on the device, 2 finished, 3 failed                      */
    int32_t iterations;   /* iterations run (< total_iter when the tolerance was reached)           */
    int32_t hbm;          /* 1: occupancy kept in HBM                                              */
    int32_t pad_;
    double submit_ms;     /* host clock, ms since the server was created                            */
    double admit_ms;
    double finish_ms;     /* step end at which the finish was collected                             */
    double device_ms;     /* device clock from the server's start to the request's final sort       */
    int64_t rounds, evals, accepts;
    int64_t device_bytes; /* arena bytes the request held                                           */
} hea_request_info;

typedef struct hea_server_status {
    int32_t queued, running, finished_unread, slots_free;
    int64_t arena_free_bytes, arena_bytes;
    int64_t rounds, evals, accepts, finished; /* cumulative */
    double busy_ms;                           /* sum of the step launches' device time */
    int32_t launches, smem_bytes;
} hea_server_status;

typedef struct hea_server hea_server;
int hea_server_create(const hea_server_config *config, hea_server **out);
int hea_server_submit(hea_server *server, const hea_problem *problem, const hea_params *params, double tolerance,
                      int32_t priority, int64_t *out_id);
int hea_server_submit_lattice(hea_server *server, int32_t lattice, int32_t cell, int32_t shell_set,
                              int32_t num_types, int32_t num_shells, const int32_t *species, const double *weight,
                              const double *target_sro, const hea_params *params, double tolerance,
                              int32_t priority, int64_t *out_id);
int hea_server_step(hea_server *server, int32_t *out_finished);
/* Ids of requests that finished (or failed) since the last call, up to cap. */
int hea_server_take_finished(hea_server *server, int64_t *ids, int32_t cap, int32_t *count);
int hea_server_result(hea_server *server, int64_t id, uint8_t *out_occ, double *out_fitness,
                      hea_request_info *info);
int hea_server_info(hea_server *server, int64_t id, hea_request_info *info);
int hea_server_status_get(hea_server *server, hea_server_status *status);
void hea_server_destroy(hea_server *server);

/*
 * Component entry points (host buffers), one launch each, used to check the
 * pieces of the search against the CPU restatement.
 *
 * hea_generate: `count` random occupancies of generation `generation`
 *   (accelerate.cpp:218-252 / accelerate.cu:912-935), with their pair counts
 *   [count][S][T][T] and f2 [count].
 * hea_recount: pair counts and f2 of given occupancies (accelerate.cpp:370-399,
 *   :118-180).
 * hea_local_search: the local parallel search on `count` occupancies in place
 *   (accelerate.cpp:601-694 / accelerate.cu:626-731) as local search number
 *   mc_call of a run; optional trace of accepted swaps (trace_cap records and
 *   count snapshots per occupancy, trace_len [count]).
 */
int hea_generate(const hea_problem *problem, uint64_t seed, uint32_t generation, int32_t count, uint8_t *out_occ,
                 int32_t *out_counts, double *out_f2);
int hea_recount(const hea_problem *problem, int32_t count, const uint8_t *occ, int32_t *out_counts, double *out_f2);
int hea_local_search(const hea_problem *problem, uint64_t seed, uint32_t mc_call, int32_t count, int32_t tasks,
                     int32_t depth, int64_t max_rounds, uint8_t *occ, int32_t *out_counts, double *out_f2,
                     int64_t *out_rounds, hea_accept_record *trace, int32_t *trace_counts, int64_t trace_cap,
                     int64_t *trace_len);

/*
 * Allocation-free form of hea_recount (same arguments, same results; NULL
 * out_counts or out_f2 are skipped, as there).  It has no counterpart in the
 * reference.  It is for callers that cannot allocate device memory -- a
 * process whose GPU memory is reserved up front by another allocator, or code
 * that must not trigger cudaMalloc's device-wide synchronisation -- and it
 * never calls cudaMalloc or cudaFree: all its device buffers live in one
 * static device array of HEA_NOALLOC_SCRATCH_BYTES, which every GPU that
 * loads the library holds until the process exits.  Every call looks up that
 * array's address in the context current on the calling thread (so a device
 * reset or another current context on the device is safe); the first call in
 * a context loads the library's device code there, so make it before any
 * stream capture.  Inputs whose raw and padded neighbour tables plus `count`
 * occupancy rows, counts and f2 exceed the array are rejected with
 * HEA_ERR_UNSUPPORTED.  All calls share the array and find the previous
 * call's contents there (the error flag is cleared and the counts rebuilt
 * from zero every call): calls that overlap on the GPU (from two host
 * threads) race.
 */
#define HEA_NOALLOC_SCRATCH_BYTES (16u << 20)
int hea_recount_noalloc(const hea_problem *problem, int32_t count, const uint8_t *occ, int32_t *out_counts,
                        double *out_f2);

/*
 * Neighbour table of a perfect cubic supercell built on the device, in the
 * site numbering and shell order of pyhea/lattice/lattice.py:146-323
 * (ids sorted within each shell).  lattice: 0 = FCC, 1 = BCC.  shell_set:
 * 0 = the reference's shells (FCC 12/6/12 with the third shell at sqrt(2) a,
 * lattice.py:283-287; BCC 8/6/12), 1 = FCC 12/6/24 with the third shell at
 * sqrt(3/2) a (BCC unchanged).  out_nbor [N][sum sizes] with N = 4 cell^3
 * (FCC) or 2 cell^3 (BCC); out_shell_sizes [3].  Pass out_nbor = NULL to
 * query the sizes only.
 */
int hea_build_neighbors(int32_t lattice, int32_t cell, int32_t shell_set, int32_t *out_nbor,
                        int32_t *out_shell_sizes, int32_t *out_num_sites);

#ifdef __cplusplus
}
#endif

#endif /* HEA_CUDA_H */
