// tcb_batch.h — internal interface of the batched form, shared with the
// served form: a batch holds up to `cap` stream slots that may be filled
// and emptied between steps; one step advances the listed slots by one
// frame each in shared CTU-engine launches.
#pragma once
#include <vector>

#include <cuda_runtime.h>

#include "../../include/tcodec_b200.h"

struct tcb_batch;

namespace tcb {

tcb_batch *batch_new(int cap);
void batch_free(tcb_batch *b);
// Puts an encoder (moved onto the batch's stream) into the first free
// slot; returns the slot or -1 when the batch is full.
int batch_attach(tcb_batch *b, tc_encoder_t *e);
// Destroys the slot's encoder (after the batch's stream is idle).
void batch_detach(tcb_batch *b, int slot);
tc_encoder_t *batch_slot(tcb_batch *b, int slot);
cudaStream_t batch_stream(tcb_batch *b);
void batch_set_graphs(tcb_batch *b, bool on);
// Runs one frame of every slot in `part` (each already planned with
// plan_input / plan_flush); packets[slot] / status[slot] receive the result.
tc_error_t batch_run(tcb_batch *b, const std::vector<int> &part, tc_packet_t *packets, int *status);

}  // namespace tcb
