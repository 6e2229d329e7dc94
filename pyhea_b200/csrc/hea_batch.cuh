// hea_batch.cuh -- many independent structures in one persistent kernel.
//
// Every structure runs the same search as the plain path (hea_search.cuh) with
// its own constants, tables, population pools and Philox key, so its result
// is bit-identical to searching it alone.  The work of all structures is a
// queue of jobs in HBM:
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
// (pyhea/cpp/accelerate.cpp:305-330, :693) -- and appends the next phase's jobs.
// Structures are ranked by work (sites x solutions x iterations) into
// kBatchLevels queues; a CTA takes the next published job of the highest
// level that has one, so the largest structures -- the longest chains of
// dependent phases -- advance first, a few at a time (their neighbour tables
// then stay in L2), and the smaller ones fill the gaps.  Each
// queue's slot count is known in advance (P (2I + 1) per structure); a CTA
// exits once every slot of every queue has been taken.  Waits are bounded by
// wall time; on expiry the kernel sets an error flag and every CTA returns.
#pragma once
#include <cstdint>

#include "hea_search.cuh"

namespace hea {

enum BatchJobKind : int32_t { kJobGen0 = 0, kJobGenMc = 1, kJobMc2 = 2 };

struct BatchJob {
    int32_t structure, kind, index, iter;
    int32_t ready;  // 1 once the fields above are visible
    int32_t pad_[3];
};

// Kernel instance of a structure: species count and shell layout.
enum BatchLayout : int32_t { kLayBcc = 0, kLayFccTrue = 1, kLayRt1 = 2, kLayRt2 = 3, kLayRt3 = 4 };

struct BatchStruct {
    SearchConst c;
    const int4 *nbor;
    uint8_t *occ;
    int32_t *cnt;
    double *f2;
    int32_t *order;    // [2P] slot ids
    int32_t *scratch;  // [2P] sort scratch
    int32_t P, Q, D, I;
    int64_t max_rounds;
    int32_t T, layout, level, pad_;
};

static_assert(sizeof(SearchConst) % 8 == 0 && alignof(SearchConst) >= 8, "SearchConst copied as 8-byte words");

struct BatchState {
    int32_t remaining;  // jobs of the current phase not finished
    int32_t phase;
};

constexpr int kBatchLevels = 16;

struct BatchQueue {
    unsigned long long head;   // slots taken
    unsigned long long tail;   // slots reserved by producers
    unsigned long long total;  // slots this queue will ever hold
    unsigned long long base;   // first slot of this queue in the job array
};

struct BatchCtl {
    BatchQueue q[kBatchLevels];
    unsigned long long stats[4];  // rounds, evals, accepts, finished structures
    int32_t error;                // 1: a wait ran out of time
    int32_t pad_;
    unsigned long long wait_limit_ns;
    unsigned long long start_ns;  // device clock when the phase-0 jobs were queued
};

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

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

// Append `n` jobs of one kind for structure s to queue `level` (block-wide;
// thread 0 reserves the slots).
__device__ __forceinline__ void enqueue_jobs(BatchJob *jobs, BatchCtl *ctl, int level, int s, int kind, int iter,
                                             int n, unsigned long long *base_sh)
{
    if (threadIdx.x == 0) *base_sh = ctl->q[level].base + atomicAdd(&ctl->q[level].tail, (unsigned long long)n);
    __syncthreads();
    const unsigned long long base = *base_sh;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        BatchJob &j = jobs[base + i];
        j.structure = s;
        j.kind = kind;
        j.index = i;
        j.iter = iter;
        __threadfence();
        atomicExch(&j.ready, 1);
    }
    __syncthreads();
}

// Thread 0: take the next reserved slot of the highest level that has one.
// Returns the slot, or -1 when every slot of every queue is taken (or on error).
__device__ __forceinline__ long long claim_job(BatchCtl *ctl)
{
    const unsigned long long t0 = global_ns();
    for (;;) {
        bool left = false;
        for (int l = 0; l < kBatchLevels; ++l) {
            volatile BatchQueue *q = &ctl->q[l];
            unsigned long long h = q->head;
            if (h < q->total) left = true;
            while (h < q->tail) {
                const unsigned long long old = atomicCAS(&ctl->q[l].head, h, h + 1);
                if (old == h) return (long long)(q->base + h);
                h = old;
            }
        }
        if (!left) return -1;
        if (*(volatile int32_t *)&ctl->error) return -1;
        if (global_ns() - t0 > ctl->wait_limit_ns) {
            atomicExch(&ctl->error, 1);
            return -1;
        }
        __nanosleep(256);
    }
}

// Initial jobs of every structure (phase 0); one CTA per structure.
__global__ void batch_seed_kernel(BatchStruct *structs, BatchState *states, BatchJob *jobs, BatchCtl *ctl)
{
    __shared__ unsigned long long base;
    const int s = blockIdx.x;
    if (s == 0 && threadIdx.x == 0) ctl->start_ns = global_ns();
    const BatchStruct &d = structs[s];
    if (threadIdx.x == 0) {
        states[s].phase = 0;
        states[s].remaining = d.I > 0 ? 2 * d.P : d.P;
    }
    for (int i = threadIdx.x; i < 2 * d.P; i += blockDim.x) d.order[i] = i;
    __syncthreads();
    enqueue_jobs(jobs, ctl, d.level, s, kJobGen0, 0, d.P, &base);
    if (d.I > 0) enqueue_jobs(jobs, ctl, d.level, s, kJobGenMc, 0, d.P, &base);
}

// One job of a structure with species count T and layout L.  Shared memory:
// occ5 (occ_stride + 16) | per-warp counts | swap records.
#ifndef HEA_BATCH_AHEAD
#define HEA_BATCH_AHEAD true  // whole-row loads before use (the batch kernel has 128 registers per thread)
#endif
template <int T, class L>
__device__ __noinline__ void batch_job(const SearchConst &c, const BatchStruct &d, const BatchJob &job, uint8_t *smem,
                                       unsigned long long *stats)
{
    constexpr int S = L::S, NC = S * T * T, NCP = mc_ncount_pad(NC);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    uint8_t *occ5 = smem;
    int32_t *cnt_all = reinterpret_cast<int32_t *>(smem + c.occ_stride + 16);
    SwapRecord *rec = reinterpret_cast<SwapRecord *>(cnt_all + nwarps * NCP);
    const int P = d.P;
    const int pos = job.index;
    const int slot = __ldcg(d.order + (job.kind == kJobGenMc ? P + pos : pos));
    uint8_t *gocc = d.occ + (size_t)slot * c.occ_stride;
    int32_t *gcnt = d.cnt + (size_t)slot * NC;

    double cur;
    if (job.kind == kJobMc2) {
        stage_occupancy<true>(c, gocc, occ5);
        for (int x = lane; x < NC; x += 32) cnt_all[warp * NCP + x] = __ldcg(gcnt + x);
        __syncthreads();
        if (threadIdx.x == 0) occ5[c.num_sites] = 0;
        cur = __ldcg(d.f2 + slot);
        __syncthreads();
    } else {
        const uint32_t generation = job.kind == kJobGen0 ? 0u : (uint32_t)(job.iter + 1);
        generate_occupancy<T>(c, (uint32_t)pos, generation, occ5, job.kind == kJobGen0 ? gocc : nullptr);
        if (threadIdx.x == 0) occ5[c.num_sites] = 0;
        __syncthreads();
        block_recount<T, S>(c, d.nbor, occ5, cnt_all);  // copy 0; ends with a barrier
        cur = fitness_of_counts<T, S>(c, cnt_all);
        if (job.kind == kJobGen0) {
            if (warp == 0)
                for (int x = lane; x < NC; x += 32) gcnt[x] = cnt_all[x];
            if (threadIdx.x == 0) d.f2[slot] = cur;
            return;
        }
        for (int x = lane; x < NC; x += 32)
            if (warp) cnt_all[warp * NCP + x] = cnt_all[x];
        __syncthreads();
    }
    const uint32_t call = job.kind == kJobMc2 ? (uint32_t)(2 * job.iter + 1) : (uint32_t)(2 * job.iter);
    const uint32_t stream = (call << 16) | (uint32_t)pos;
    const McTally t =
        mc_rounds<T, L, HEA_BATCH_AHEAD>(c, d.nbor, occ5, cnt_all, rec, stream, cur, d.Q, d.D, d.max_rounds,
                                         McTrace{nullptr, nullptr, 0});
    unstage_occupancy(c, occ5, gocc);
    if (warp == 0)
        for (int x = lane; x < NC; x += 32) gcnt[x] = cnt_all[x];
    add_tally(t, stats);
    if (threadIdx.x == 0) d.f2[slot] = t.f2;
}

template <int T>
__device__ __forceinline__ void batch_dispatch_t(const SearchConst &c, const BatchStruct &d, const BatchJob &job,
                                                 uint8_t *smem, unsigned long long *stats)
{
    switch (d.layout) {
    case kLayBcc: batch_job<T, Shells<2, 2, 3>>(c, d, job, smem, stats); break;
    case kLayFccTrue: batch_job<T, Shells<3, 2, 6>>(c, d, job, smem, stats); break;
    case kLayRt1: batch_job<T, RuntimeShells<1>>(c, d, job, smem, stats); break;
    case kLayRt2: batch_job<T, RuntimeShells<2>>(c, d, job, smem, stats); break;
    default: batch_job<T, RuntimeShells<3>>(c, d, job, smem, stats); break;
    }
}

#ifndef HEA_BATCH_THREADS
#define HEA_BATCH_THREADS 256
#endif

// The persistent kernel: CTAs claim job slots in order until every slot is
// done.  Dynamic shared memory: the largest structure's occupancy + 16 +
// per-warp counts + swap records; the job's constants (1.9 KB) are copied to
// static shared memory, which still leaves two CTAs per SM for 108 000-site
// structures.
__global__ void __launch_bounds__(HEA_BATCH_THREADS, 2)
    batch_kernel(const BatchStruct *__restrict__ structs, BatchState *states, BatchJob *jobs, BatchCtl *ctl,
                 unsigned long long *finish_ns)
{
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ BatchJob job;
    __shared__ int stop, last, phase;
    __shared__ unsigned long long base;
    __shared__ __align__(16) SearchConst c;  // this job's constants: fitness tables read from shared memory
    for (;;) {
        if (threadIdx.x == 0) {
            stop = 0;
            const long long h = claim_job(ctl);
            if (h < 0) {
                stop = 1;
            } else {
                volatile int32_t *ready = &jobs[h].ready;
                const unsigned long long t0 = global_ns();
                while (*ready == 0) {  // the producer reserved this slot and is filling it
                    if (*(volatile int32_t *)&ctl->error || global_ns() - t0 > ctl->wait_limit_ns) {
                        atomicExch(&ctl->error, 1);
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
                }
            }
        }
        __syncthreads();
        if (stop) break;
        // this job's structure: read-only during the launch
        const BatchStruct &d = structs[job.structure];
        {  // 8-byte words: SearchConst holds doubles, so it is 8-byte aligned and sized
            const int2 *src = reinterpret_cast<const int2 *>(&d.c);
            int2 *dst = reinterpret_cast<int2 *>(&c);
            for (int x = threadIdx.x; x < (int)(sizeof(SearchConst) / 8); x += blockDim.x) dst[x] = __ldg(src + x);
        }
        __syncthreads();
        switch (d.T) {
        case 2: batch_dispatch_t<2>(c, d, job, smem, ctl->stats); break;
        case 3: batch_dispatch_t<3>(c, d, job, smem, ctl->stats); break;
        case 4: batch_dispatch_t<4>(c, d, job, smem, ctl->stats); break;
        case 5: batch_dispatch_t<5>(c, d, job, smem, ctl->stats); break;
        default: batch_dispatch_t<6>(c, d, job, smem, ctl->stats); break;
        }
        __threadfence();  // every writer orders its results before the completion count
        __syncthreads();
        if (threadIdx.x == 0) {
            last = atomicSub(&states[job.structure].remaining, 1) == 1;
            if (last) {
                __threadfence();
                phase = __ldcg(&states[job.structure].phase);
            }
        }
        __syncthreads();
        if (!last) continue;
        // phase transition of this structure
        const int s = job.structure, P = d.P, I = d.I, k = phase;
        if (k == 0 && I == 0) {  // generation 0 only: the reference returns it unsorted
            if (threadIdx.x == 0) {
                finish_ns[s] = global_ns() - ctl->start_ns;
                atomicAdd(&ctl->stats[3], 1ull);
            }
            continue;
        }
        if (k > 0) block_stable_sort(d.order, d.f2, P, d.scratch);      // survivors after their search
        if (k < I) block_stable_sort(d.order, d.f2, 2 * P, d.scratch);  // merge of iteration k
        if (k == I) {
            if (threadIdx.x == 0) {
                finish_ns[s] = global_ns() - ctl->start_ns;
                atomicAdd(&ctl->stats[3], 1ull);
            }
            continue;
        }
        if (threadIdx.x == 0) {
            states[s].phase = k + 1;
            states[s].remaining = (k + 1 < I) ? 2 * P : P;
            __threadfence();
        }
        __syncthreads();
        enqueue_jobs(jobs, ctl, d.level, s, kJobMc2, k, P, &base);
        if (k + 1 < I) enqueue_jobs(jobs, ctl, d.level, s, kJobGenMc, k + 1, P, &base);
    }
}

}  // namespace hea
