// Entry points of the one-sync proof pipeline used by vg_session_prove.
// They are internal to the library (the public C ABI is include/virgo_b200.h):
// every call only enqueues work on the context stream; results stay on the
// device or land in pinned host memory that is valid after the stream is
// synchronised.
#pragma once
#include "virgo_b200.h"

// ---- GKR (gkr.cu) ----
// Deferred mode on: rounds and v_res write records of 9 values on the device
// (round: the 3 sums, then the 6 folded values when one pair remained;
// v_res: the value) instead of returning them; records are numbered in call
// order from 0.
int vg_gkr_defer(vg_gkr *g, int on);
// phase2_init whose v_u = fold of the previous record's V pair at r_last,
// plus addend, is formed on the device.
int vg_gkr_phase2_init_deferred(vg_gkr *g, const vg_fe *r_u, int length_u, vg_fe r_last, vg_fe addend);
// Enqueues the copy of all records to pinned host memory (*host, 9 * *n values).
int vg_gkr_records(vg_gkr *g, const vg_fe **host, int *n);
// Phase round sequences issued from a captured CUDA graph so far (replays)
// and captured so far (captures), counted over the object's life.
void vg_gkr_graph_counts(const vg_gkr *g, long long *replays, long long *captures);

// Sumcheck tables without a circuit: vg_gkr_round (deferred) over tables the
// caller fills.  vg_gkr_tables_begin flushes the rounds still queued, hands
// out the AV and AM tables (n entries, to be written before the next round)
// and takes V (n entries, read in place by the first round).  Records as in
// deferred mode, numbered from the last rewind; vg_gkr_destroy frees.
int vg_gkr_tables_create(vg_ctx *ctx, long max_n, int max_records, vg_gkr **out);
int vg_gkr_tables_reserve(vg_gkr *g, long max_n, int max_records);
int vg_gkr_tables_rewind(vg_gkr *g);
int vg_gkr_tables_begin(vg_gkr *g, const vg_fe *V, long n, vg_fe **AV, vg_fe **AM);
const vg_fe *vg_gkr_records_dev(const vg_gkr *g);
int vg_gkr_record_count(const vg_gkr *g);

// vg_fft_gkr_prove in two halves: the launch enqueues the whole side proof
// on the object's context stream; the finish waits for it and checks the
// messages (so other work can be launched in between).
int vg_fft_gkr_launch(vg_fft_gkr *f, int lg, unsigned seed);
int vg_fft_gkr_finish(vg_fft_gkr *f, vg_fft_gkr_stats *st, vg_fe *msgs, vg_fe *vals);
// Raises the largest size the object proves to max_lg (buffers from the
// stream-ordered pool, no device-wide synchronisation).
int vg_fft_gkr_reserve(vg_fft_gkr *f, int max_lg);

// The evaluation's input layer read from `input` (device, layer-0 width)
// instead of the circuit's own values; null goes back to the circuit's.
int vg_gkr_set_input(vg_gkr *g, const vg_fe *input);
// Layer-0 values from n input-gate u values on the device (read through int32
// as the circuit build does), zero up to width; enqueued on c's stream.
int vg_input_values(vg_ctx *c, const int64_t *dev_u, long n, long width, vg_fe *out);
// Host-to-device copy on c's stream (pageable sources through the context's
// pinned ring; a pageable source may be reused on return).
int vg_h2d_staged(vg_ctx *c, void *dst, const void *src, size_t bytes);
// Work enqueued on waiter's stream from now on waits for the work enqueued so
// far on signaler's.
int vg_ctx_wait_for(vg_ctx *waiter, vg_ctx *signaler);

// Replaces c's stream by one of the device's highest priority (drains the
// old one first).
int vg_ctx_raise_priority(vg_ctx *c);

// Grows a device buffer from the stream-ordered pool on c's stream.
int vg_ctx_grow_dev(vg_ctx *c, void **p, size_t *cap, size_t bytes);

// vg_eq_table without the final synchronisation.
int vg_eq_table_async(vg_ctx *c, const vg_fe *r, int log_len, vg_fe *pub);

// ---- commitment + FRI + queries (commit.cu) ----
struct vg_pc_results {
    const vg_fe *inner;          // sampled <l, q>, compared with the sumcheck claim
    const vg_fe *all_sum;        // 65
    const vg_digest *roots;      // 2 + nlevels: l, h, then every FRI level
    const vg_fe *final_cw;       // last FRI level, 65 slices of n_final, slice-major
    long n_final;
    const vg_fe *qvals;          // nq x 130: the 65 value pairs of each query
    const vg_digest *qpaths;     // nq x 32: siblings bottom-up, then the leaf
};
// Mask length M the private mask is padded to (poly_commit.h:66-70).
long vg_pc_mask_len(int log_len, long n_pri_mask);
// The whole commitment of one proof: RS encodings of the private input and of
// the public eq table, the virtual oracle, every FRI fold (challenges fri_r),
// all leaf chains and Merkle trees batched, the query answers for
// (which, pos) as in vg_pc_query_batch, and the copies of every result into
// pinned memory (out points there).
int vg_pc_prove_deferred(vg_pc *pc, const vg_fe *priv, int log_len, const vg_fe *pri_mask, long n_pri_mask,
                         const vg_fe *pub, const vg_fe *pub_mask, long n_pub_mask, const vg_fe *fri_r, int nlevels,
                         int nq, const int *which, const long *pos, vg_pc_results *out);
