/*
 * sa_b200_batch.h -- C ABI of the batched persistent engine.
 *
 * A batch holds many independent disorder instances of mixed shape (2D, 2D
 * open-x, 3D; any even L), each an ensemble of `nslots` 64-replica systems
 * sharing one coupling set -- the reference's parallel_tempering<gpu_sys>
 * (src/parallel_tempering.hpp) over systems built the way its driver builds
 * them (src/main_gpu.cu:251-277): set_seed(seed_J); init_J(); set_seed(seed);
 * init_rand(); so every slot starts from the same spins and draws the same
 * per-site Philox stream, and the slots share J.
 *
 * One persistent kernel advances every instance: a CTA takes an instance from
 * a work queue and runs all requested sweeps of all its slots, with the
 * replica exchange of src/parallel_tempering.hpp:81-115 done on the device:
 * the exchange pair and uniform of every step come from the reference's own
 * generator (std::mt19937(123), uniform_int_distribution<int>(0, n-2),
 * uniform_real_distribution<double>(0,1)) on the host, converted to an exact
 * integer accept interval for dE (valid for h = 0, which a batch requires).
 *
 * Anneal schedules: an instance may instead carry a temperature schedule
 * (nslots = 1): one temperature per `sweeps_per_step` sweeps, with the running
 * maximum of -H per replica tracked on the device (src/annealing.hpp:67-100).
 */
#ifndef SA_B200_BATCH_H
#define SA_B200_BATCH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sa_batch* sa_batch_t;

/* Empty batch on the current device. */
int sa_batch_create(sa_batch_t* out);
int sa_batch_destroy(sa_batch_t b);

/* A temperature ladder (sorted ascending internally, as the PT constructor
 * does, src/parallel_tempering.hpp:193-218). */
int sa_batch_add_ladder(sa_batch_t b, const double* T, int n, int* ladder_id);
/* A temperature schedule for annealing instances: T[k] holds for sweeps
 * [k*sweeps_per_step, (k+1)*sweeps_per_step); the last entry holds after. */
int sa_batch_add_schedule(sa_batch_t b, const double* T, int nsteps, int sweeps_per_step,
                          int* schedule_id);
/* An instance. Exactly one of ladder_id / schedule_id is >= 0. */
int sa_batch_add_instance(sa_batch_t b, int lattice, int L, int ladder_id, int schedule_id,
                          uint64_t seed_J, uint64_t seed, int* instance_id);
/* Allocates the spin / coupling pools, generates J and the initial spins on
 * the device and uploads the tables. No instance may be added afterwards. */
int sa_batch_finalize(sa_batch_t b);

/* Energy histograms, before finalize: every `stride` sweeps (0 = off) every
 * slot of every parallel-tempering instance is measured (before the
 * exchange) and its 64 replica energies are binned on the device; bin b of a
 * slot counts E = 2b - nbonds. Needs the resident kernel. */
int sa_batch_set_histograms(sa_batch_t b, int stride);
/* Histogram of one slot: *nbins = nbonds + 1; out (host) may be NULL. */
int sa_batch_histogram(sa_batch_t b, int instance, int slot, int32_t* out, long cap, long* nbins);
/* Kernel choice, before finalize: 0 (default) keeps every instance whose
 * spins fit in the shared memory of a cluster of <= 16 CTAs resident there for
 * a whole launch and runs the rest in the global-memory kernel, except that a
 * single-slot 3D anneal of L >= 40 with the GPU nearly to itself runs wide
 * (every column of a colour a lane group anywhere on the GPU, three launches
 * per sweep); 1 runs every instance in the global-memory kernel; 2 is 0
 * without the wide form. */
int sa_batch_set_kernel(sa_batch_t b, int kernel);
/* Kernel launches one sa_batch_run issues (one per launch group). */
int sa_batch_launches_per_run(sa_batch_t b, int* n);
/* Launch shapes of the resident kernel. A bucket is (lattice, L, slots); its
 * shape is seven int32: lattice, L, slots, C (CTAs per instance cluster), SL
 * (slots per lane: 1, or 2 for an even slot count), warps per block, and 1
 * for the high-register form of the two-slot 3D walk. No counterpart in the
 * reference (it launches one system per kernel with a fixed 16x16 / 8x8x8
 * block); the shapes replace the engine's own launch heuristics.
 * sa_tuning_table: the built-in table (measured on a B200 by
 * simulated_annealing_b200/autotune.py); out == NULL reports the count.
 * sa_batch_set_tuning: before finalize, use these n entries instead (n = 0:
 * the heuristics only; n < 0: back to the built-in table). Buckets without an
 * entry, and batches whose clusters were spread over idle SMs, keep the
 * heuristic shapes. sa_batch_set_spread(b, 0): never spread (full-batch
 * shapes even for a few instances). sa_batch_instance_shape: after finalize,
 * the seven values an instance runs with (C = 0: the global-memory kernel,
 * C = -1: the wide form). */
int sa_tuning_table(int32_t* out, int cap, int* n);
int sa_batch_set_tuning(sa_batch_t b, const int32_t* entries, int n);
int sa_batch_set_spread(sa_batch_t b, int on);
int sa_batch_instance_shape(sa_batch_t b, int id, int32_t* out);
/* Per launch group (one shape per group, each on its own stream): with
 * sa_batch_set_group_timing(b, 1) before finalize, sa_batch_group_times
 * gives, for the last sa_batch_run, each group's five int32 (lattice, L,
 * instances, C, warps) and the milliseconds from the run's start to the
 * group's end -- the tail of the slowest group. info / ms may be NULL;
 * *n receives the group count. No counterpart in the reference. */
int sa_batch_set_group_timing(sa_batch_t b, int on);
int sa_batch_group_times(sa_batch_t b, int32_t* info, float* ms, int cap, int* n);
/* Sweeps between exchange attempts (the PT template's `steps`; default 1). */
int sa_batch_set_exchange_interval(sa_batch_t b, int sweeps_per_exchange);
/* Anneal instances: measure every `stride` sweeps (0 = never; default 1) and
 * fold the result into the per-replica running maximum of -H. */
int sa_batch_set_measure_stride(sa_batch_t b, int stride);
/* Record every exchange (pair, mask) of every PT instance, up to `capacity`
 * exchanges per instance. */
int sa_batch_record_exchanges(sa_batch_t b, long capacity);

/* Advance every unfinished instance by up to `nsweeps` sweeps (anneal
 * instances stop at the end of their schedule). Asynchronous on the batch's
 * stream; the launch and its tables are prepared on the host first. */
int sa_batch_run(sa_batch_t b, long nsweeps);
int sa_batch_sync(sa_batch_t b);
int sa_batch_set_stream(sa_batch_t b, void* stream);
/* Number of sites processed per sweep over the whole batch (sum N*nslots). */
int sa_batch_site_slots(sa_batch_t b, long long* site_slots);
int sa_batch_num_instances(sa_batch_t b, int* n);

/* Read-back (synchronous). Spins in the reference's row-major layout. */
int sa_batch_get_spins(sa_batch_t b, int instance, int slot, uint64_t* s);
int sa_batch_get_J(sa_batch_t b, int instance, uint64_t* jx, uint64_t* jy, uint64_t* jz);
/* Exact E per replica bit of one slot (sum over bonds of +-1). */
int sa_batch_measure(sa_batch_t b, int instance, int slot, int64_t* E);
/* Accepted replica count and attempts per adjacent pair (nslots-1 each). */
int sa_batch_acceptance(sa_batch_t b, int instance, int64_t* accepted, int64_t* attempts);
/* Recorded exchanges of one instance: pairs[count], masks[count]. */
int sa_batch_exchanges(sa_batch_t b, int instance, int* pairs, uint64_t* masks, long cap,
                       long* count);
/* Energies of every slot of every instance, into HOST memory E (pinned for
 * speed): E[off(i) + slot*64 + j], off(i) = 64 * sum of nslots of instances
 * before i. Asynchronous on the batch stream (sync before reading E). */
int sa_batch_energies(sa_batch_t b, int64_t* E);
/* Number of int64 values sa_batch_energies writes (64 * sum of nslots). */
int sa_batch_energy_count(sa_batch_t b, long long* n);
/* Acceptance counters of all pairs of all instances (instance-major), into
 * host memory; asynchronous like sa_batch_energies. */
int sa_batch_acceptance_all(sa_batch_t b, int64_t* accepted, int64_t* attempts);
int sa_batch_num_pairs(sa_batch_t b, long long* n);
/* Host->device bytes the last sa_batch_run copied (its exchange decisions). */
int sa_batch_last_h2d_bytes(sa_batch_t b, long long* n);
/* Anneal instances: running maximum of -H per replica (int64[64]) and the
 * number of sweeps done. */
int sa_batch_anneal_result(sa_batch_t b, int instance, int64_t* Emax, long* sweeps_done);
/* Sweeps done by an instance so far. */
int sa_batch_sweeps_done(sa_batch_t b, int instance, long* sweeps_done);

/* ---- serving: continuous batching of anneal requests ------------------------
 * No reference counterpart: the reference runs one system per process
 * (src/main.cpp). A server owns device pools sized from budget_bytes and
 * admits a request (lattice, L, coupling seed, spin/RNG seed, schedule T[nsteps]
 * of sweeps_per_step sweeps each) only when the pools have room; otherwise
 * sa_serve_submit returns SA_ERR_BUDGET and the caller retries after
 * collecting results. Each sa_serve_run call advances every active request by
 * up to nsweeps sweeps in one set of launches (the batch kernels); requests
 * join at the next call. A request's result depends only on its own
 * parameters, never on what runs beside it. sa_serve_poll lists finished
 * requests; sa_serve_result copies one out (after sa_serve_sync) and frees it.
 */
typedef struct sa_serve* sa_serve_t;

int sa_serve_create(size_t budget_bytes, int max_requests, sa_serve_t* out);
int sa_serve_destroy(sa_serve_t s);
int sa_serve_set_stream(sa_serve_t s, void* stream);
int sa_serve_submit(sa_serve_t s, int lattice, int L, uint64_t seed_J, uint64_t seed, const double* T, int nsteps,
                    int sweeps_per_step, int64_t* id);
int sa_serve_run(sa_serve_t s, long nsweeps);
int sa_serve_sync(sa_serve_t s);
int sa_serve_poll(sa_serve_t s, int64_t* ids, int cap, int* n);
/* Emax: running max of -H per replica over the measurements (int64[64]);
 * Elast: last measured -H (int64[64], may be NULL); spins: final row-major
 * spin words (N of them, may be NULL). Frees the request. */
int sa_serve_result(sa_serve_t s, int64_t id, int64_t* Emax, int64_t* Elast, uint64_t* spins);
int sa_serve_active(sa_serve_t s, int* n, long long* free_words);

#ifdef __cplusplus
}
#endif
#endif /* SA_B200_BATCH_H */
