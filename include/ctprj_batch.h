/*
 * ctprj_batch.h -- many slices of different geometries in one launch.
 *
 * No single counterpart in the reference, which projects one configured slice
 * per gpuPrj() call (prj/gpuPrj.cu:887-1047) and reconfigures with setup()
 * between geometries; a batch replaces that loop.  Each slice keeps the exact
 * semantics of ctprj_forward / ctprj_backward for its geometry (results are
 * identical); the whole batch runs as one batched quad-image pass plus one persistent
 * forward kernel, or one persistent backprojection kernel, and can be captured
 * in CUDA graphs.  Launch shapes are chosen by ctprj_batch_autotune.
 */
#ifndef CTPRJ_BATCH_H
#define CTPRJ_BATCH_H

#include "ctprj.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ctprj_batch ctprj_batch;

/* One plan per slice on `device` (-1: current). */
int ctprj_batch_create(const ctprj_geometry *geoms, int nslices, int device, ctprj_batch **batch);
void ctprj_batch_destroy(ctprj_batch *batch);

/* Device buffers of every slice (host arrays of nslices device pointers):
 * forward d_imgs[i] (n*n) -> d_sinos[i] (np*prjWidth); backward d_bsinos[i] ->
 * d_bimgs[i].  Either pair may be NULL.  Drops captured graphs. */
int ctprj_batch_bind(ctprj_batch *batch, const float *const *d_imgs, float *const *d_sinos,
                     const float *const *d_bsinos, float *const *d_bimgs);

/* Batched forward projection / backprojection of all bound slices on
 * `stream` (through the captured graph when there is one). */
int ctprj_batch_forward(ctprj_batch *batch, void *stream);
int ctprj_batch_backward(ctprj_batch *batch, void *stream);

/* Capture the forward and the backward launch sequences into CUDA graphs,
 * replayed by the two calls above until the next bind or autotune. */
int ctprj_batch_capture(ctprj_batch *batch, void *stream);

/* Time the candidate launch shapes on the bound buffers (both directions bound)
 * and keep the fastest; with cache_path, reuse and record choices keyed by the
 * device and the geometries.  Synchronises `stream`. */
int ctprj_batch_autotune(ctprj_batch *batch, void *stream, const char *cache_path);

/* Streaming backprojection: the persistent kernel starts before the inputs
 * exist and backprojects slice i once the host has published it by setting
 * flag i != 0 (after its sinogram is on the device), in host-mapped flags from
 * ctprj_stream_flags_create.  A slice not published within timeout_s (at most
 * 60 s) of a block starting to wait for it is given up: its output is left
 * untouched, status[i] = 1 (status: nslices ints, may be NULL) and the call
 * returns CTPRJ_ETIMEOUT; the device stays usable.  Synchronises `stream`. */
int ctprj_stream_flags_create(int n, int **host_flags, int **dev_flags);
void ctprj_stream_flags_destroy(int *host_flags);
int ctprj_batch_stream_backward(ctprj_batch *batch, const int *dev_flags, double timeout_s,
                                int *status, void *stream);

/* Text of the current launch configuration. */
int ctprj_batch_config(ctprj_batch *batch, char *buf, int len);

#ifdef __cplusplus
}
#endif

#endif /* CTPRJ_BATCH_H */
