/*
 * ctprj_noalloc.h -- forward projection without any device allocation.
 *
 * No counterpart in the reference: the reference allocates its device buffers
 * in setup() (prj/gpuPrj.cu:850-851).  This entry point is for callers that
 * cannot call cudaMalloc -- code running inside another framework's memory
 * pool or allocator, real-time loops that must not block on allocation, or
 * embedders that have reserved the whole GPU.  It calls no cudaMalloc, no
 * cudaFree and no allocating library routine; its scratch (the forward pass's
 * quad image -- the eight symmetric copies of each pixel, twice the image's
 * size -- and the ray tables, about 8.5 MiB) is a set of file-scope device
 * arrays that every GPU loading the library holds until the process exits.
 */
#ifndef CTPRJ_NOALLOC_H
#define CTPRJ_NOALLOC_H

#include "ctprj.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Same result as ctprj_plan_create + ctprj_forward for `geom`, on the current
 * device: d_sino[np*prjWidth] = A d_img[n*n], enqueued on `stream`.
 * Limits: n <= 1024, prjWidth <= 4096, prjFull <= 8192; larger geometries
 * return CTPRJ_ERANGE.  All calls share the scratch arrays: calls that overlap
 * on the GPU (other streams, other host threads) race and must be serialised by
 * the caller.  The first call on a device looks up the arrays' device
 * addresses; make it before any stream capture.  Those addresses are kept until
 * the process exits, so a caller must not reset the device (cudaDeviceReset)
 * and then call again.  A call on a stream that is being captured returns
 * CTPRJ_EINVAL: the table uploads read static host buffers that every later
 * call overwrites. */
int ctprj_forward_noalloc(const ctprj_geometry *geom, const float *d_img, float *d_sino,
                          void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CTPRJ_NOALLOC_H */
