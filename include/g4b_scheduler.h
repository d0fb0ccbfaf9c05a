/*
 * g4b_scheduler.h - streaming batch scheduler in front of the transport engine.
 *
 * Replaces the host side of OpticalBatchScheduler
 * (include/g4go/optical/geant4/OpticalBatchScheduler.hpp:32-93,
 *  src/optical/geant4/OpticalBatchScheduler.cpp):
 *
 *   OpticalBatchScheduler(config) + BeginRun()   -> g4b_scheduler_create
 *   Submit(OpticalSubmission) -> future           -> g4b_scheduler_submit -> ticket
 *   future.get()                                  -> g4b_scheduler_wait(ticket)
 *   EndRun()                                      -> g4b_scheduler_end_run
 *   RunStatistics() / BatchStatistics()           -> g4b_scheduler_statistics
 *   ~OpticalBatchScheduler()                      -> g4b_scheduler_destroy
 *
 * Any number of producer threads (the Geant4 workers) submit one event's
 * gensteps at a time; one transport thread owned by the scheduler collects
 * submissions into batches (target photon count, event cap, collection
 * timeout: OpticalBatchScheduler.cpp:462-509), transports them and hands each
 * event its own detections and statistics after the batch/event consistency
 * checks of CompleteBatch (:243-446).
 *
 * Unlike the reference, which completes a batch before it collects the next
 * one (:579-593), the scheduler drives several engine handles (one stream and
 * one set of pinned staging each) and keeps that many batches in flight: it
 * collects and stages batch k+1 while the GPU transports batch k, so k+1's
 * persistent kernel starts on the SMs that k's drained warps leave, and it
 * splits k's output per event while the later batches run. Every photon's history depends only on its
 * RNG counters, so the batches' composition changes no detection.
 * serial = 1 restores the reference's order on one handle.
 *
 * Statuses and g4b_scheduler_last_error follow g4b.h. The reference's
 * exceptions map as there: invalid_argument for inconsistent submissions,
 * runtime_error ("queue is not ready", "queue is stopping") as G4B_ERR_LOGIC,
 * and a failure inside the transport thread (a CUDA error, a failed
 * consistency check, duplicate event IDs in one batch) fails every request of
 * the run and every later submission, as ProcessBatches does (:595-617).
 */
#ifndef G4B_SCHEDULER_H
#define G4B_SCHEDULER_H

#include "g4b.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The batching fields of PhotonTransportConfig
 * (include/g4go/optical/PhotonTransportConfig.hpp:31-37); zero selects the
 * reference's default. */
typedef struct g4b_scheduler_config {
    uint32_t abi_version;                  /* must be G4B_ABI_VERSION */
    uint32_t target_photons_per_batch;     /* 0 -> 1,000,000 */
    uint32_t max_events_per_batch;         /* 0 -> 10,000 */
    uint32_t max_queued_photons;           /* 0 -> 2,000,000 */
    uint32_t max_queued_submissions;       /* 0 -> 1,024 */
    uint32_t batch_collection_timeout_ms;  /* 0 -> 10 */
    uint32_t enable_performance_diagnostics; /* 1: time queue waits and flattening, as the reference does */
    uint32_t serial;                       /* 1: the reference's order (retire batch k before collecting k+1); 0: pipelined */
    uint32_t batches_in_flight;            /* pipelined: engine handles, and batches on the GPU at once; 0 -> 8, at most 8 */
    uint32_t reserved[7];
} g4b_scheduler_config;

/* PhotonBatchStatistics (OpticalBatchScheduler.hpp:20-32) plus the scheduler
 * fields of PhotonTransportPerformance (PhotonTransport.hpp:106-108) and the
 * summed engine performance of the batches. */
typedef struct g4b_batch_statistics {
    uint64_t batch_count;
    uint64_t event_count;
    uint64_t photon_count;
    uint64_t max_batch_photon_count;
    uint64_t max_batch_event_count;
    uint64_t queue_high_water_mark;
    uint64_t min_batch_photon_count;
    uint64_t total_queue_wait_count;
    double scheduler_input_wait_ms;     /* transport thread waiting for submissions */
    double scheduler_gpu_wait_ms;       /* transport thread waiting for a batch to finish */
    double scheduler_queue_wait_ms;     /* submissions waiting in the queue (summed) */
    double scheduler_batch_flatten_ms;
    uint64_t scheduler_batch_flatten_bytes;
    uint64_t overlapped_batch_count;    /* batches launched while another one was on the GPU */
    g4b_performance performance;        /* engine performance, summed over batches */
} g4b_batch_statistics;

typedef struct g4b_scheduler g4b_scheduler;

/* A transport the scheduler drives in place of its own engine handle: the
 * five calls keep the contracts of g4b_enqueue, g4b_poll_oldest,
 * g4b_query_oldest, g4b_complete and g4b_last_error. They are made from the
 * scheduler's transport thread only. */
typedef struct g4b_transport_ops {
    void* context;
    int (*enqueue)(void* context, const g4b_optical_emission* emissions, uint32_t emission_count,
                   const uint32_t* event_ids, uint32_t event_count, const uint32_t* emission_event_indices);
    int (*poll)(void* context, int* ready);
    int (*query)(void* context, uint64_t* detection_count, uint32_t* event_count);
    int (*complete)(void* context, g4b_output* output);
    const char* (*last_error)(void* context);
} g4b_transport_ops;

/* Constructor + BeginRun (OpticalBatchScheduler.cpp:20-120): starts the
 * transport thread, which creates the engine handles from engine_config (two,
 * or one when serial), sets the scene on each (copied before this call
 * returns) and then waits for submissions. Returns the engine's status if
 * either step fails. Detections come back per event in flattened-photon order
 * when engine_config->ordered_detections is set. */
int g4b_scheduler_create(const g4b_config* engine_config, const g4b_scene* scene,
                         const g4b_scheduler_config* config, g4b_scheduler** out_scheduler);

/* The same scheduler over caller-supplied transports: ops[0..ops_count) (1 to
 * 4; each one more lets one more batch be in flight) are copied, and their
 * contexts must outlive the scheduler. batches_in_flight is ignored. */
int g4b_scheduler_create_with_transport(const g4b_transport_ops* ops, uint32_t ops_count,
                                        const g4b_scheduler_config* config, g4b_scheduler** out_scheduler);

/* Submit (OpticalBatchScheduler.cpp:144-218): queues one event's gensteps
 * (copied before the call returns) and returns its ticket. photon_count must
 * equal the sum of the emissions' photon counts; every emission carries
 * event_id. source_statistics (generated/captured counts from Geant4) may be
 * NULL. Blocks while the queue holds max_queued_submissions submissions or
 * adding this one would exceed max_queued_photons (a single submission larger
 * than the limit is admitted into an empty queue). A submission with no
 * photons completes at once. Thread-safe. */
int g4b_scheduler_submit(g4b_scheduler* scheduler, uint32_t event_id, const g4b_optical_emission* emissions,
                         uint32_t emission_count, uint64_t photon_count, const g4b_statistics* source_statistics,
                         uint64_t* ticket);

/* future.get(): waits up to timeout_ms (negative: without limit; 0: poll) for
 * the ticket's event and fills output like g4b_complete: its detections in
 * the batch's flattened-photon order, one event_statistics record, the
 * event's statistics (source fields merged with the transport's terminal
 * fields as CompleteBatch does, :265-314) and a zero performance record.
 * G4B_ERR_TIMEOUT if not ready yet; G4B_ERR_CAPACITY with the needed counts
 * if the caller's buffers are too small (the ticket stays). Success or a
 * failed transport releases the ticket; a released or unknown ticket is
 * G4B_ERR_INVALID_ARGUMENT. Thread-safe. */
int g4b_scheduler_wait(g4b_scheduler* scheduler, uint64_t ticket, int64_t timeout_ms, g4b_output* output);

/* EndRun (OpticalBatchScheduler.cpp:122-142): refuses new submissions,
 * transports everything already queued, then stops the transport thread and
 * releases the engine. Tickets stay waitable until g4b_scheduler_destroy. */
int g4b_scheduler_end_run(g4b_scheduler* scheduler);

/* RunStatistics / BatchStatistics: totals so far. Either pointer may be NULL. */
int g4b_scheduler_statistics(g4b_scheduler* scheduler, g4b_statistics* run, g4b_batch_statistics* batch);

/* Replays a recorded run through the scheduler, the way the Geant4 workers
 * submit it: event i (ID event_ids[i], gensteps
 * emissions[emission_offsets[i] .. emission_offsets[i+1])) is submitted by
 * producer thread i % producers, in order, each thread keeping at most
 * `window` events outstanding and collecting their results (detections are
 * counted, not kept). *detections is the total returned, *seconds the wall
 * time from the first submission to the last result. No counterpart in the
 * reference; it replays captured gensteps and measures the scheduler with
 * native producers. */
int g4b_scheduler_replay(g4b_scheduler* scheduler, const g4b_optical_emission* emissions,
                         const uint64_t* emission_offsets, const uint32_t* event_ids, uint32_t event_count,
                         uint32_t producers, uint32_t window, uint64_t* detections, double* seconds);

/* End the run if it is still going and free everything. */
int g4b_scheduler_destroy(g4b_scheduler* scheduler);

/* Message of the last failed scheduler call on this thread. Never NULL. */
const char* g4b_scheduler_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* G4B_SCHEDULER_H */
