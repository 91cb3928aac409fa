// Internal interface of the batched executor, used by the request server.
#pragma once
#include "amhj_host.h"

namespace amj {

int normalize_batch_opts(const amj_batch_opts *in, amj_batch_opts *o);
// enqueue a run of the batch (no waiting); batch_done polls, batch_collect waits
int batch_launch(amj_batch *b, const amj_batch_opts &o);
bool batch_done(amj_batch *b);
// forget the submitted queries but keep the device and pinned buffers
void batch_clear(amj_batch *b);
int batch_collect(amj_batch *b, uint64_t *counts, uint64_t *checksums, amj_batch_stats *stats);
// device bytes a run of the submitted queries would allocate
uint64_t batch_estimate_bytes(const amj_batch *b, const amj_batch_opts &o);

}  // namespace amj
