/*
 * bgt_capi.h -- C ABI of the B200 thinning library (libbgt.so).
 *
 * Plain C types only: host or device pointers, sizes, integer status codes.
 * Every entry point returns BGT_OK (0) or a positive bgt_status; the message
 * of the last failure on the calling thread is available from
 * bgt_last_error().  Nothing here exits the process or reads stdin.
 *
 * Pixel data is row-major with x fastest: 2D data[y*width + x],
 * 3D data[(z*height + y)*width + x].  Foreground follows the reference's
 * binarisation: 2D (unsigned int)v > 0 (2D/CUDA_DeviceHelperFunctions.cuh:101),
 * 3D int(v) > 0 (3D/CenterlineExtraction.cpp:44).  Thinned outputs are 0/1 in
 * the input's pixel type.
 */
#ifndef BGT_CAPI_H
#define BGT_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Pixel types of the reference's explicit instantiations
 * (2D/LibThinning2D.cu:134-143, 2D/CenterlineExtraction.cpp:146-155). */
typedef enum bgt_dtype {
    BGT_U8 = 0,   /* unsigned char */
    BGT_I8 = 1,   /* signed char */
    BGT_CHAR = 2, /* char */
    BGT_U16 = 3,  /* unsigned short */
    BGT_I16 = 4,  /* short */
    BGT_U32 = 5,  /* unsigned int */
    BGT_I32 = 6,  /* int */
    BGT_F32 = 7,  /* float */
    BGT_F64 = 8,  /* double */
    BGT_BOOL = 9  /* bool (one byte) */
} bgt_dtype;

typedef enum bgt_status {
    BGT_OK = 0,
    BGT_ERR_ARG = 1,      /* invalid argument (null pointer, bad size or dtype) */
    BGT_ERR_CUDA = 2,     /* a CUDA runtime call failed */
    BGT_ERR_NOMEM = 3,    /* device or host allocation failed */
    BGT_ERR_TIMEOUT = 4,  /* a bounded device wait gave up (status word set by a kernel) */
    BGT_ERR_LIMIT = 5,    /* an instance hit the pass cap or a size limit */
    BGT_ERR_STATE = 6     /* call out of order (e.g. run before finalize) */
} bgt_status;

typedef struct bgt_ctx bgt_ctx;     /* device, stream, resident scratch */
typedef struct bgt_batch bgt_batch; /* a set of images/volumes thinned together */

/* ---- context ---------------------------------------------------------- */
/* Binds `device`; creates a private stream.  Resident device scratch grows on
 * demand and is kept until bgt_ctx_destroy. */
int bgt_ctx_create(int device, bgt_ctx **out);
int bgt_ctx_destroy(bgt_ctx *ctx);
/* Use a caller stream (cudaStream_t passed as void*) for subsequent calls;
 * NULL restores the context's own stream. */
int bgt_ctx_set_stream(bgt_ctx *ctx, void *stream);
const char *bgt_last_error(void);
int bgt_version(void);

/* ---- drop-in thinning (host buffers, synchronous) ---------------------
 * Replace Thinning2D<T> (2D/LibThinning2D.h:14-15) and Thinning3D<T>
 * (3D/LibThinning3D.h:14-15): `in` and `out` are host arrays of `dtype`
 * with width*height(*depth) elements; any size >= 1 is accepted. */
int bgt_thin2d(bgt_ctx *ctx, int dtype, const void *in, int width, int height, void *out);
int bgt_thin3d(bgt_ctx *ctx, int dtype, const void *in, int width, int height, int depth, void *out);

/* ---- device-resident thinning (device buffers, stream-ordered) -------- */
int bgt_thin2d_device(bgt_ctx *ctx, int dtype, const void *d_in, int width, int height, void *d_out);
int bgt_thin3d_device(bgt_ctx *ctx, int dtype, const void *d_in, int width, int height, int depth,
                      void *d_out);

/* ---- thinning without device allocation --------------------------------
 * No counterpart in the reference.  For callers that must not allocate
 * device memory (a plugin inside a host application that owns all device
 * memory through its own pool, a real-time loop that cannot afford an
 * allocation's implicit synchronisation): thins one 2D image of `dtype`
 * from d_in to d_out (device buffers, width*height pixels) on `stream`
 * (a cudaStream_t, NULL = legacy default stream) of `device` (the caller's
 * current device is restored on return), synchronising the stream once
 * per pass,
 * using only an 8 MiB scratch array compiled into the library (kept by
 * every GPU that loads it until the process exits).  Images whose packed
 * form does not fit (beyond about 4096 x 4096) are rejected with
 * BGT_ERR_LIMIT.  No cudaMalloc or cudaFree is called.  Calls share the
 * array: they are serialised by a process-wide lock and each returns after
 * its work on `stream` finished; work arranged to overlap on the GPU would
 * race on the array.  The first call on a device looks up the array's
 * address; make it before any stream capture. */
int bgt_thin2d_device_noalloc(int device, int dtype, const void *d_in, int width, int height, void *d_out,
                              void *stream);

/* ---- centreline extraction (host buffers, synchronous) ----------------
 * Replace CenterlineExtraction<T> (2D/CenterlineExtraction.h:25-28,
 * 3D/CenterlineExctraction.h:26-29): thinning, segment extraction, pruning
 * of end segments with at most max_segment_length points, moving-average
 * smoothing with half-width smoothing_span, CSR output.  *out_x, *out_y
 * (*out_z), *out_idx are allocated with malloc (free with bgt_free);
 * out_idx has nsegs+1 entries, out_idx[nsegs] = number of points. */
int bgt_centerline2d(bgt_ctx *ctx, int dtype, const void *in, int width, int height, int max_segment_length,
                     int smoothing_span, float **out_x, float **out_y, unsigned int **out_idx,
                     unsigned int *nsegs);
int bgt_centerline3d(bgt_ctx *ctx, int dtype, const void *in, int width, int height, int depth,
                     int max_segment_length, int smoothing_span, float **out_x, float **out_y, float **out_z,
                     unsigned int **out_idx, unsigned int *nsegs);
void bgt_free(void *p);

/* MATLAB column order of centreline output, as the reference's MEX gateways
 * build their cell arrays (2D/Matlab2DThinning.cpp:163-175,
 * 3D/Matlab3DThinning.cpp:157-171): segment i becomes an ssize x dims
 * column-major double matrix whose columns are y, x (and z), ssize =
 * idx[i+1] - idx[i].  The matrices are written back to back into out
 * (dims * idx[nsegs] doubles; segment i starts at out + dims * idx[i]).
 * z is ignored (may be null) when dims == 2.  Host memory, no device work. */
int bgt_matlab_segments(int dims, unsigned int nsegs, const float *x, const float *y, const float *z,
                        const unsigned int *idx, double *out);

/* ---- segment extraction on the device -------------------------------
 * Replace ExtractSegmentsV<T> (2D/ExtractSegments.h:16-17,
 * 3D/ExtractSegments.h:21-22) on a thinned 0/1 image already in device
 * memory.  Outputs (host, malloc'ed, free with bgt_free): per segment its
 * start offset (nseg+1 entries) and is_end_segment flag; per point x, y (z)
 * as int16.  Segments come in the reference's emission order. */
int bgt_segments2d_device(bgt_ctx *ctx, int dtype, const void *d_img, int width, int height, int32_t **start,
                          uint8_t **is_end, int16_t **px, int16_t **py, int *nseg, int *npts);
int bgt_segments3d_device(bgt_ctx *ctx, int dtype, const void *d_vol, int width, int height, int depth,
                          int32_t **start, uint8_t **is_end, int16_t **px, int16_t **py, int16_t **pz, int *nseg,
                          int *npts);

/* ---- batched thinning ---------------------------------------------------
 * Hundreds of images/volumes of uneven size thinned together by one
 * persistent launch fed by a device-side queue of (instance, tile) work
 * items, each instance converging on its own.  Usage: create, add shapes,
 * finalize (allocates, picks tile configurations), set device input/output
 * pointers, run (any number of times), destroy. */
int bgt_batch_create(bgt_ctx *ctx, bgt_batch **out);
int bgt_batch_destroy(bgt_batch *b);
/* cfg < 0 lets the autotuner choose; returns the instance id in *id */
int bgt_batch_add2d(bgt_batch *b, int width, int height, int cfg, int *id);
int bgt_batch_add3d(bgt_batch *b, int width, int height, int depth, int cfg, int *id);
int bgt_batch_finalize(bgt_batch *b);
/* Reuse without allocation: reserve a device pool once (before the first
 * finalize); reset drops the instances (keeping the pool) so the batch can
 * be refilled and finalized again; a set of instances that does not fit
 * the reserved pool fails finalize with BGT_ERR_LIMIT. */
int bgt_batch_reserve(bgt_batch *b, size_t bytes);
int bgt_batch_reset(bgt_batch *b);
/* Cap the persistent engine's CTAs (0 = a full wave of the device) so
 * batches running on several streams share the SMs. */
int bgt_batch_set_grid(bgt_batch *b, int ctas);
int bgt_batch_set_io(bgt_batch *b, int id, int dtype, const void *d_in, void *d_out);
/* mode 0: persistent engine (optionally replayed as a CUDA graph when
 * use_graph != 0); mode 1: plain path, one launch per pass per instance with
 * a host readback of the change flag after every pass; mode 2: the same
 * passes with the loop on the device (a CUDA graph with one conditional
 * WHILE node per instance, built on the first run and replayed; use_graph is
 * ignored), so no pass waits for the host. */
int bgt_batch_run(bgt_batch *b, int mode, int use_graph);
/* per-instance passes run and whether it converged (1) / hit the cap (-1) */
int bgt_batch_instance_stats(bgt_batch *b, int id, int *passes, int *converged, int *cfg);
/* device bytes held by the batch */
int bgt_batch_device_bytes(bgt_batch *b, size_t *bytes);
/* work of the last run, summed over instances: tiles processed (skipped
 * tiles excluded) and packed core words processed (one read + one write of
 * 4 bytes each is the algorithmic traffic of a word-pass) */
int bgt_batch_work(bgt_batch *b, unsigned long long *tiles, unsigned long long *words);
/* device milliseconds of the last engine run's stages (CUDA events on the
 * batch's stream): pack, engine (the thinning kernels), unpack */
int bgt_batch_stage_ms(bgt_batch *b, float *pack_ms, float *engine_ms, float *unpack_ms);
/* The engine stage split: the resident kernel (instances thinned inside
 * one CTA's shared memory, large images as bands of CTAs) and the tile-ring
 * engine after it (instances the resident kernel does not take, volumes
 * whose non-empty bricks did not fit). */
int bgt_batch_engine_ms(bgt_batch *b, float *resident_ms, float *rings_ms);
/* Engine choice for the next finalize: 0 = resident kernel wherever an
 * instance fits (default), 1 = tile rings only.  Instances added with an
 * explicit configuration (cfg >= 0) always use the tile rings. */
int bgt_batch_set_engine(bgt_batch *b, int mode);
/* Plan of instance id after finalize: *resident = 1 when the resident
 * kernel takes it, *bands = the CTAs a 2D image is cut into (0 for rings). */
int bgt_batch_plan(bgt_batch *b, int id, int *resident, int *bands);
/* Timeline of the resident kernel's work items in the last run (no
 * reference counterpart; for tracing load balance): per item, in the order
 * taken, its instance, band, start and end in ns from the earliest start
 * (device global timer) and the SM that ran it.  *n = number of items; at
 * most cap are written.  Synchronises the batch's stream. */
int bgt_batch_res_trace(bgt_batch *b, int *n, int *inst, int *band, long long *t0_ns, long long *t1_ns, int *sm,
                        int cap);

/* ---- serving -------------------------------------------------------------
 * A request loop over the batch engine.  Requests (2D frames: depth 1; 3D
 * volumes: depth > 1) are submitted from any host thread with host buffers
 * (pinned memory keeps the copies asynchronous) that must stay valid until
 * the request completes.  A dispatcher thread admits waiting requests into
 * free slots of their lane (frames: high-priority streams; volumes:
 * low-priority streams) and launches them while earlier launches still run
 * (continuous batching).  Device memory is one arena of hbm_budget_bytes,
 * allocated at creation and resident; each launch holds a block of it sized
 * from its requests (staging + batch pool) until its outputs are back in
 * host memory, and a request waits until the arena has room for it (volumes
 * leave a guard for one launch of frames).  A request larger than its lane
 * may ever hold is rejected at submit with BGT_ERR_LIMIT.  Latency = submit
 * to output in host memory. */
typedef struct bgt_server bgt_server;
int bgt_server_create(int device, size_t hbm_budget_bytes, bgt_server **out);
int bgt_server_submit(bgt_server *s, int dtype, const void *host_in, int width, int height, int depth,
                      void *host_out, unsigned long long *ticket);
/* completed requests since the last poll (ticket, latency in ms, status) */
int bgt_server_poll(bgt_server *s, unsigned long long *tickets, double *latency_ms, int *status, int cap, int *n);
int bgt_server_drain(bgt_server *s, double timeout_s);
/* lane 0 = frames, 1 = volumes: latency percentiles, Mvoxel/s, completed count */
int bgt_server_stats(bgt_server *s, int lane, double *p50_ms, double *p99_ms, double *mvox_per_s,
                     unsigned long long *completed);
int bgt_server_reset_stats(bgt_server *s);
/* arena bytes held by launches in flight, the arena's size, and requests
 * waiting for admission */
int bgt_server_memory(bgt_server *s, size_t *used, size_t *budget, unsigned long long *waiting);
int bgt_server_destroy(bgt_server *s);

/* ---- tile configurations and the autotuner's table --------------------
 * The autotuner (begputhinning_b200/tune.py) times the configurations on
 * sample instances of each size class and records the winner here; batches
 * finalized afterwards use it for instances added with cfg < 0. */
int bgt_tune_class(int dims, int width, int height, int depth);
int bgt_tune_set(int dims, int cls, int cfg); /* cfg < 0 restores the default */
int bgt_tune_get(int dims, int cls, int *cfg);

/* Number of configurations for dims (2 or 3) and their ids. */
int bgt_cfg_list(int dims, int *ids, int cap, int *n);
/* k = subiterations per pass, tw/th/tz = core tile extent (words, rows, planes) */
int bgt_cfg_describe(int id, int *dims, int *k, int *tw, int *th, int *tz, int *smem_bytes);

/* Self-test of the device rules (no reference counterpart): the deletable
 * set of direction dir (2D 0..3 = N,S,E,W; 3D 0..5 = U,N,E,D,S,W) over every
 * neighbourhood of a foreground centre, 32 neighbourhoods per word.
 * Neighbour i (2D: N,NE,E,SE,S,SW,W,NW; 3D: the 26 neighbours in (dz,dy,dx)
 * order, centre skipped) is bit i of the neighbourhood number n; n lives in
 * bit n%32 of word n/32.  d_out: 8 words (2D) or 2^21 words (3D) of device
 * memory.  Synchronises the stream. */
int bgt_rule_table(int dims, int dir, uint32_t *d_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif
