// hea_batch.cuh -- the job engine: many independent structures searched by one
// persistent kernel.  It serves both the batch API (hea_batch_*: a fixed set
// of structures in one graph-captured launch) and the serving loop
// (hea_server_*: structures admitted while others run, in time slices).
//
// Every structure runs the same search as the plain path (hea_search.cuh) with
// its own constants, tables, population pools and Philox key, so its result
// is bit-identical to searching it alone, whatever else shares the GPU.  Its
// work is a sequence of phases of jobs:
//
//   phase 0        P x GEN0 (generation 0 of the population) and, when I > 0,
//                  P x GENMC(0) (generation 1 of the new population, then its
//                  local search, mc_call 0)
//   phase k, 1..I  P x MC2(k-1) (local search of the survivors, mc_call
//                  2(k-1)+1) and, when k < I, P x GENMC(k) (generation k+1,
//                  local search with mc_call 2k)
//
// The CTA that finishes the last job of a structure's phase runs the phase
// transition itself -- stable sort of the survivors, then the merge
// (pyhea/cpp/accelerate.cpp:305-330, :693) -- and appends the next phase's
// jobs.  With a tolerance, a local search also ends once its f2 is at or
// below it, and the structure ends once the best f2 after a survivors' sort
// is (the search of the population generated meanwhile is dropped).
//
// Jobs live in ring queues, one per priority level, whose head and tail only
// grow; a CTA takes the next reserved job of the highest level that has one
// and waits for the producer's sequence number in the slot.  A ring needs
// room for the jobs of one phase of every structure at its level (at most
// 2P each), since a phase is queued only after the previous one finished.
//
// A launch ends when no structure is active or, for the time slices of the
// serving loop, at its deadline: CTAs stop taking jobs, and a local search
// that sees the deadline stops at the end of its round, saves its state
// (occupancy, counts, f2) to HBM and queues a continuation that resumes at
// the next round with the same rejection count -- the same proposals follow,
// so the result does not depend on where the slices fell.  Waits are bounded
// by wall time since the last finished job; on expiry the kernel sets an
// error flag and every CTA returns.
//
// Occupancy in HBM (`hbm`, the default: proposals are scored from the site
// histograms, so a search reads the occupancy only for its draws): a job
// converts the row to 5*species in place (reads through L2, so no stale L1
// line of another SM's writes is used; the conversion rewrites every byte this
// CTA later reads), searches it through L1, and converts it back.  Otherwise
// the row is staged in the launch's shared memory.
#pragma once
#include <cstdint>

#include "hea_search.cuh"

namespace hea {

enum BatchJobKind : int32_t { kJobGen0 = 0, kJobGenMc = 1, kJobMc2 = 2 };

struct BatchJob {
    int32_t structure, kind, index, iter;
    int32_t seq;     // low 32 bits of (ring position + 1), written after the other fields
    int32_t resume;  // 1: continue a stopped local search at round0 with miss0 rejections
    int32_t round0, miss0;
};
static_assert(sizeof(BatchJob) == 32, "BatchJob layout");

// Kernel instance of a structure: species count and shell layout.
enum BatchLayout : int32_t {
    kLayBcc = 0, kLayFccTrue = 1, kLayRt1 = 2, kLayRt2 = 3, kLayRt3 = 4, kLayImp1 = 5, kLayImp2 = 6, kLayImp3 = 7
};

struct BatchStruct {
    SearchConst c;
    const int4 *nbor;
    uint8_t *occ;
    int32_t *cnt;
    double *f2;
    int32_t *order;    // [2P] slot ids
    int32_t *scratch;  // [2P] sort scratch
    uint4 *hist;       // [2P][N] site histograms
    const uint32_t *nbmask;
    int32_t P, Q, D, I;
    int64_t max_rounds;
    double tol2;  // tolerance on f2 (< 0: none): local searches and the structure end once reached
    int32_t T, layout, level, hbm;
};

static_assert(sizeof(SearchConst) % 8 == 0 && alignof(SearchConst) >= 8, "SearchConst copied as 8-byte words");

struct BatchState {
    int32_t remaining;  // jobs of the current phase not finished
    int32_t phase;      // at the end: the iterations run
    int32_t done;       // 1 once the structure's search ended
    int32_t pad_;
    unsigned long long tally[3];  // rounds, evals, accepts of this structure
};

constexpr int kBatchLevels = 16;

struct BatchQueue {
    unsigned long long head;  // jobs taken
    unsigned long long tail;  // jobs reserved by producers
    unsigned long long cap;   // ring slots
    unsigned long long base;  // first slot of this ring in the job array
};

struct BatchCtl {
    BatchQueue q[kBatchLevels];
    unsigned long long stats[4];  // rounds, evals, accepts, finished structures
    int32_t error;                // 1: a wait ran out of time, 2: a ring slot was overwritten
    int32_t active;               // structures seeded and not finished
    unsigned long long wait_limit_ns;
    unsigned long long start_ns;     // device time origin of finish times
    unsigned long long deadline_ns;  // device time after which no job starts (0: none)
    unsigned long long progress_ns;  // device time of the last finished job
};

// Stable ascending order of order[0, count) by f2 (rank counting); block-wide,
// barriers inside.  scratch holds `count` ints.  Reads go through L2: the
// values were written by other CTAs of the same launch.
__device__ __forceinline__ void block_stable_sort(int32_t *order, const double *f2, int count, int32_t *scratch)
{
    for (int i = threadIdx.x; i < count; i += blockDim.x) scratch[i] = __ldcg(order + i);
    __syncthreads();
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
        const double fi = __ldcg(f2 + __ldcg(scratch + i));
        int r = 0;
        for (int j = 0; j < count; ++j) {
            const double fj = __ldcg(f2 + __ldcg(scratch + j));
            r += (fj < fi) || (fj == fi && j < i);
        }
        order[r] = __ldcg(scratch + i);
    }
    __threadfence();
    __syncthreads();
}

__device__ __forceinline__ BatchJob &ring_slot(BatchJob *jobs, const BatchQueue &q, unsigned long long h)
{
    return jobs[q.base + h % q.cap];
}

// Append `n` fresh jobs of one kind for structure s to ring `level`
// (block-wide; thread 0 reserves the positions).
__device__ __forceinline__ void enqueue_jobs(BatchJob *jobs, BatchCtl *ctl, int level, int s, int kind, int iter,
                                             int n, unsigned long long *first_sh)
{
    if (threadIdx.x == 0) *first_sh = atomicAdd(&ctl->q[level].tail, (unsigned long long)n);
    __syncthreads();
    const unsigned long long first = *first_sh;
    const BatchQueue &q = ctl->q[level];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const unsigned long long h = first + i;
        BatchJob &j = ring_slot(jobs, q, h);
        j.structure = s;
        j.kind = kind;
        j.index = i;
        j.iter = iter;
        j.resume = 0;
        j.round0 = 0;
        j.miss0 = 0;
        __threadfence();
        atomicExch(&j.seq, (int32_t)(uint32_t)(h + 1));
    }
    __syncthreads();
}

// Thread 0: the continuation of a stopped local search.
__device__ __forceinline__ void enqueue_resume(BatchJob *jobs, BatchCtl *ctl, int level, const BatchJob &job,
                                               int64_t round0, int miss0)
{
    const unsigned long long h = atomicAdd(&ctl->q[level].tail, 1ull);
    BatchJob &j = ring_slot(jobs, ctl->q[level], h);
    j.structure = job.structure;
    j.kind = job.kind;
    j.index = job.index;
    j.iter = job.iter;
    j.resume = 1;
    j.round0 = (int32_t)round0;
    j.miss0 = miss0;
    __threadfence();
    atomicExch(&j.seq, (int32_t)(uint32_t)(h + 1));
}

// Thread 0: take the next reserved job of the highest level that has one.
// Returns its slot and expected sequence number, or -1 when no structure is
// active, the deadline has passed, or on error.
__device__ __forceinline__ long long claim_job(BatchCtl *ctl, unsigned long long deadline, int32_t *seq)
{
    const unsigned long long t0 = global_ns();
    for (;;) {
        if (*(volatile int32_t *)&ctl->active <= 0 || *(volatile int32_t *)&ctl->error) return -1;
        const unsigned long long now = global_ns();
        if (deadline && now >= deadline) return -1;
        for (int l = 0; l < kBatchLevels; ++l) {
            volatile BatchQueue *q = &ctl->q[l];
            unsigned long long h = q->head;
            while (h < q->tail) {
                const unsigned long long old = atomicCAS(&ctl->q[l].head, h, h + 1);
                if (old == h) {
                    *seq = (int32_t)(uint32_t)(h + 1);
                    return (long long)(q->base + h % q->cap);
                }
                h = old;
            }
        }
        const unsigned long long prog = *(volatile unsigned long long *)&ctl->progress_ns;
        const unsigned long long since = prog > t0 ? prog : t0;  // another SM's clock read may be ahead of ours
        if (now > since && now - since > ctl->wait_limit_ns) {
            atomicExch(&ctl->error, 1);
            return -1;
        }
        __nanosleep(256);
    }
}

// Phase-0 jobs of structures list[0, gridDim.x) (all structures when list is
// NULL); one CTA per structure.
__global__ void batch_seed_kernel(const BatchStruct *structs, const int32_t *list, BatchState *states, BatchJob *jobs,
                                  BatchCtl *ctl)
{
    __shared__ unsigned long long first;
    const int s = list ? list[blockIdx.x] : (int)blockIdx.x;
    const BatchStruct &d = structs[s];
    if (threadIdx.x == 0) {
        BatchState &st = states[s];
        st.remaining = d.I > 0 ? 2 * d.P : d.P;
        st.phase = 0;
        st.done = 0;
        st.tally[0] = st.tally[1] = st.tally[2] = 0;
        __threadfence();
        atomicAdd(&ctl->active, 1);
    }
    for (int i = threadIdx.x; i < 2 * d.P; i += blockDim.x) d.order[i] = i;
    __syncthreads();
    enqueue_jobs(jobs, ctl, d.level, s, kJobGen0, 0, d.P, &first);
    if (d.I > 0) enqueue_jobs(jobs, ctl, d.level, s, kJobGenMc, 0, d.P, &first);
}

struct JobEnd {
    int32_t yielded, round, miss;
};

// One job of a structure with species count T and layout L.  Shared memory:
// [occ5 (occ_stride + 16), unless hbm] | search_smem_tail(T, S, nwarps) (delta
// table, swap records, two count buffers).
// The rounds of a job's local search in a call of their own: values the job
// needs only before and after the search stay out of the loop's registers.
template <int T, class L>
__device__ __noinline__ McTally batch_search(const SearchConst &c, const BatchStruct &d, uint8_t *occ5, int32_t *cnt2,
                                             double2 *tab, SwapRecord *rec, uint32_t stream, double cur,
                                             const McResume rs, uint4 *hist)
{
    return mc_rounds<T, L, true>(c, d.nbor, occ5, cnt2, tab, rec, stream, cur, d.Q, d.D, d.max_rounds,
                                 McTrace{nullptr, nullptr, 0}, rs, hist, d.nbmask);
}

template <int T, class L>
__device__ __noinline__ JobEnd batch_job(const SearchConst &c, const BatchStruct &d, const BatchJob &job,
                                         uint8_t *smem, unsigned long long *stats, unsigned long long *tally,
                                         unsigned long long deadline)
{
    constexpr int S = L::S, NC = S * T * T, NCP = mc_ncount_pad(NC);
    const int nwarps = blockDim.x >> 5;
    const bool hbm = d.hbm != 0;
    const int P = d.P, n = c.num_sites;
    const int pos = job.index;
    const int slot = __ldcg(d.order + (job.kind == kJobGenMc ? P + pos : pos));
    uint8_t *gocc = d.occ + (size_t)slot * c.occ_stride;
    int32_t *gcnt = d.cnt + (size_t)slot * NC;
    uint4 *hist = d.hist + (size_t)slot * c.num_sites;
    uint8_t *occ5 = hbm ? gocc : smem;
    double2 *tab = reinterpret_cast<double2 *>(hbm ? smem : smem + c.occ_stride + 16);
    SwapRecord *rec = reinterpret_cast<SwapRecord *>(tab + delta_entries(T, S));
    int32_t *cnt2 = reinterpret_cast<int32_t *>(rec + 2 * nwarps);

    double cur;
    if (job.kind == kJobMc2 || job.resume) {
        stage_occupancy<true>(c, gocc, occ5);  // in place when hbm
        for (int x = threadIdx.x; x < NC; x += blockDim.x) cnt2[x] = __ldcg(gcnt + x);
        __syncthreads();
        if (threadIdx.x == 0) occ5[n] = 0;  // sentinel
        cur = __ldcg(d.f2 + slot);  // a resumed search's running f2
    } else {
        const uint32_t generation = job.kind == kJobGen0 ? 0u : (uint32_t)(job.iter + 1);
        generate_occupancy<T>(c, (uint32_t)pos, generation, occ5, (job.kind == kJobGen0 && !hbm) ? gocc : nullptr);
        if (threadIdx.x == 0) occ5[n] = 0;
        __syncthreads();
        block_recount<T, S>(c, d.nbor, occ5, cnt2, hist);  // count buffer 0; ends with a barrier
        cur = fitness_of_counts<T, S>(c, cnt2);
        if (job.kind == kJobGen0) {
            if (hbm) unstage_occupancy(c, occ5, gocc);
            for (int x = threadIdx.x; x < NC; x += blockDim.x) gcnt[x] = cnt2[x];
            if (threadIdx.x == 0) d.f2[slot] = cur;
            return JobEnd{0, 0, 0};
        }
    }
    search_setup<T, S>(c, cnt2, tab);
    const uint32_t call = job.kind == kJobMc2 ? (uint32_t)(2 * job.iter + 1) : (uint32_t)(2 * job.iter);
    const uint32_t stream = (call << 16) | (uint32_t)pos;
    const McResume rs{job.resume ? (int64_t)job.round0 : 0, job.resume ? job.miss0 : 0, deadline, d.tol2};
    // the draws read the species from the occupancy: measured on the mixed batch, the histograms'
    // species words (draw_pair_hist) were slower for every structure size
    const McTally t = batch_search<T, L>(c, d, occ5, cnt2, tab, rec, stream, cur, rs, hist);
    unstage_occupancy(c, occ5, gocc);  // in place when hbm
    for (int x = threadIdx.x; x < NC; x += blockDim.x) gcnt[x] = cnt2[t.buf * NCP + x];
    add_tally(t, stats);
    add_tally(t, tally);
    if (threadIdx.x == 0) d.f2[slot] = t.f2;  // recomputed from the counts, or the running f2 of a yielded search
    return JobEnd{t.yielded ? 1 : 0, (int32_t)t.round_end, t.miss};
}

template <int T>
__device__ __forceinline__ JobEnd batch_dispatch_t(const SearchConst &c, const BatchStruct &d, const BatchJob &job,
                                                   uint8_t *smem, unsigned long long *stats, unsigned long long *tally,
                                                   unsigned long long deadline)
{
    switch (d.layout) {
    case kLayBcc: return batch_job<T, Shells<2, 2, 3>>(c, d, job, smem, stats, tally, deadline);
    case kLayFccTrue: return batch_job<T, Shells<3, 2, 6>>(c, d, job, smem, stats, tally, deadline);
    case kLayRt1: return batch_job<T, RuntimeShells<1>>(c, d, job, smem, stats, tally, deadline);
    case kLayRt2: return batch_job<T, RuntimeShells<2>>(c, d, job, smem, stats, tally, deadline);
    case kLayImp1: return batch_job<T, ImplicitShells<1>>(c, d, job, smem, stats, tally, deadline);
    case kLayImp2: return batch_job<T, ImplicitShells<2>>(c, d, job, smem, stats, tally, deadline);
    case kLayImp3: return batch_job<T, ImplicitShells<3>>(c, d, job, smem, stats, tally, deadline);
    default: return batch_job<T, RuntimeShells<3>>(c, d, job, smem, stats, tally, deadline);
    }
}

#ifndef HEA_BATCH_THREADS
#define HEA_BATCH_THREADS 256
#endif
#ifndef HEA_BATCH_MIN_BLOCKS
#define HEA_BATCH_MIN_BLOCKS 3  // resident CTAs per SM the register budget aims for (measured: 3 > 2, 4)
#endif

// The persistent kernel: CTAs take jobs until no structure is active or the
// launch's deadline has passed.  Dynamic shared memory: occupancy of the
// largest shared-memory structure + 16 + per-warp counts + swap records; the
// job's constants (1.9 KB) are copied to static shared memory.
__global__ void __launch_bounds__(HEA_BATCH_THREADS, HEA_BATCH_MIN_BLOCKS)
    batch_kernel(const BatchStruct *__restrict__ structs, BatchState *states, BatchJob *jobs, BatchCtl *ctl,
                 unsigned long long *finish_ns)
{
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ BatchJob job;
    __shared__ int stop, last, phase;
    __shared__ unsigned long long first;
    __shared__ __align__(16) SearchConst c;  // this job's constants: fitness tables read from shared memory
    const unsigned long long deadline = ctl->deadline_ns;  // set before the launch
    for (;;) {
        if (threadIdx.x == 0) {
            stop = 0;
            int32_t seq = 0;
            const long long h = claim_job(ctl, deadline, &seq);
            if (h < 0) {
                stop = 1;
            } else {
                volatile int32_t *vs = &jobs[h].seq;
                const unsigned long long t0 = global_ns();
                while (*vs != seq) {  // the producer reserved this position and is filling it
                    if (*(volatile int32_t *)&ctl->error || global_ns() - t0 > ctl->wait_limit_ns) {
                        atomicCAS(&ctl->error, 0, 1);
                        stop = 1;
                        break;
                    }
                    __nanosleep(64);
                }
                if (!stop) {
                    __threadfence();
                    const BatchJob *src = &jobs[h];
                    job.structure = __ldcg(&src->structure);
                    job.kind = __ldcg(&src->kind);
                    job.index = __ldcg(&src->index);
                    job.iter = __ldcg(&src->iter);
                    job.resume = __ldcg(&src->resume);
                    job.round0 = __ldcg(&src->round0);
                    job.miss0 = __ldcg(&src->miss0);
                    __threadfence();
                    if (*vs != seq) {  // reused before it was read: the ring is too small
                        atomicCAS(&ctl->error, 0, 2);
                        stop = 1;
                    }
                }
            }
        }
        __syncthreads();
        if (stop) break;
        // this job's structure: read-only while it is active
        const BatchStruct &d = structs[job.structure];
        {  // 8-byte words: SearchConst holds doubles, so it is 8-byte aligned and sized
            const int2 *src = reinterpret_cast<const int2 *>(&d.c);
            int2 *dst = reinterpret_cast<int2 *>(&c);
            for (int x = threadIdx.x; x < (int)(sizeof(SearchConst) / 8); x += blockDim.x) dst[x] = __ldg(src + x);
        }
        __syncthreads();
        unsigned long long *tally = states[job.structure].tally;
        JobEnd e;
        switch (d.T) {
        case 2: e = batch_dispatch_t<2>(c, d, job, smem, ctl->stats, tally, deadline); break;
        case 3: e = batch_dispatch_t<3>(c, d, job, smem, ctl->stats, tally, deadline); break;
        case 4: e = batch_dispatch_t<4>(c, d, job, smem, ctl->stats, tally, deadline); break;
        case 5: e = batch_dispatch_t<5>(c, d, job, smem, ctl->stats, tally, deadline); break;
        default: e = batch_dispatch_t<6>(c, d, job, smem, ctl->stats, tally, deadline); break;
        }
        __threadfence();  // every writer orders its results before the completion count
        __syncthreads();
        if (threadIdx.x == 0) {
            if (e.yielded) {
                enqueue_resume(jobs, ctl, d.level, job, e.round, e.miss);
                last = 0;
            } else {
                last = atomicSub(&states[job.structure].remaining, 1) == 1;
                atomicMax(&ctl->progress_ns, global_ns());
                if (last) {
                    __threadfence();
                    phase = __ldcg(&states[job.structure].phase);
                }
            }
        }
        __syncthreads();
        if (!last) continue;
        // phase transition of this structure
        const int s = job.structure, P = d.P, I = d.I, k = phase;
        bool finished = (k == 0 && I == 0);  // generation 0 only: the reference returns it unsorted
        if (!finished) {
            if (k > 0) block_stable_sort(d.order, d.f2, P, d.scratch);  // survivors after their search
            if (k == I)
                finished = true;
            else if (k > 0 && d.tol2 >= 0.0 && __ldcg(d.f2 + __ldcg(d.order)) <= d.tol2)
                finished = true;  // tolerance reached
            else
                block_stable_sort(d.order, d.f2, 2 * P, d.scratch);  // merge of iteration k
        }
        if (finished) {
            if (threadIdx.x == 0) {
                finish_ns[s] = global_ns() - ctl->start_ns;
                states[s].done = 1;
                __threadfence();
                atomicAdd(&ctl->stats[3], 1ull);
                atomicSub(&ctl->active, 1);
            }
            __syncthreads();
            continue;
        }
        if (threadIdx.x == 0) {
            states[s].phase = k + 1;
            states[s].remaining = (k + 1 < I) ? 2 * P : P;
            __threadfence();
        }
        __syncthreads();
        enqueue_jobs(jobs, ctl, d.level, s, kJobMc2, k, P, &first);
        if (k + 1 < I) enqueue_jobs(jobs, ctl, d.level, s, kJobGenMc, k + 1, P, &first);
    }
}

}  // namespace hea
