/*
 * pst_c.h - C ABI of the B200 static priority search tree library (libpst_b200.so).
 *
 * Plain C types only: device pointers are void*, sizes are uint64_t, streams are
 * cudaStream_t-compatible handles (NULL = the legacy default stream).  Every
 * function returns a pst_status and never throws; pst_last_error() gives the
 * calling thread's last error message.
 *
 * Each entry point names the reference interface it replaces (paths relative to
 * the reference project, arraylistnumstring/static-priority-search-tree).  The
 * reference exposes C++ class templates only; these are the calls a binding for
 * that surface binds, and the C++ facade in
 * static-priority-search-tree_b200/cpp/static-pst-gpu.h re-creates the
 * reference's template signatures on top of them.
 *
 * Point records are the reference's PointStruct layouts
 * (helpers/point-struct.h:25-33, :106-117):
 *   PST_ID_U32:  { T dim1_val; T dim2_val; uint32_t id; }  (natural alignment)
 *   PST_ID_NONE: { T dim1_val; T dim2_val; }
 * Result sets are bit-exact with the reference's StaticPSTCPUIter; their order
 * on the GPU is unspecified, as it is in the reference's GPU searches.
 */
#ifndef PST_C_H
#define PST_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *pst_stream_t;

typedef enum pst_status {
	PST_OK = 0,
	PST_ERR_INVALID = 1,     /* bad argument (null handle, dtype, sizes) */
	PST_ERR_CUDA = 2,        /* a CUDA runtime call failed, or no CUDA device */
	PST_ERR_NOMEM = 3,       /* device memory allocation failed */
	PST_ERR_CAPACITY = 4,    /* caller-provided output buffer too small */
	PST_ERR_UNSUPPORTED = 5, /* combination not supported (e.g. ids from an id-less tree) */
	PST_ERR_INTERNAL = 6,    /* a device-side consistency check failed */
	PST_ERR_BUSY = 7,        /* server queue full / request not admitted */
	PST_ERR_TIMEOUT = 8      /* a bounded wait ran out */
} pst_status;

typedef enum pst_dtype { PST_F32 = 0, PST_F64 = 1, PST_I32 = 2 } pst_dtype;
typedef enum pst_idtype { PST_ID_NONE = 0, PST_ID_U32 = 1 } pst_idtype;
/* RetType of the reference searches: IDType or the whole PointStruct. */
typedef enum pst_ret { PST_RET_IDS = 0, PST_RET_POINTS = 1 } pst_ret;
typedef enum pst_qkind { PST_Q_THREE = 0, PST_Q_LEFT = 1, PST_Q_RIGHT = 2 } pst_qkind;

/* A bound in the tree's value type. */
typedef union pst_value {
	float f32;
	double f64;
	int32_t i32;
} pst_value;

/* One query.  THREE: min1 <= dim1 <= max1 and dim2 >= min2;
 * LEFT: dim1 <= max1 and dim2 >= min2; RIGHT: dim1 >= min1 and dim2 >= min2.
 * Bounds a kind does not use are ignored. */
typedef struct pst_query {
	int32_t kind;
	int32_t reserved;
	pst_value min1, max1, min2;
} pst_query;

typedef struct pst_tree pst_tree;
typedef struct pst_batch pst_batch;

/* ------------------------------------------------------------------------- */
/* Library                                                                    */

const char *pst_last_error(void);
const char *pst_version(void);
/* sizeof the PointStruct record for (dtype, idtype); 0 for an invalid pair. */
size_t pst_point_size(pst_dtype dtype, pst_idtype idtype);

/* cudaFree of a buffer a drop-in call allocated (pst_search, pst_ips_search), for
 * bindings that do not link the CUDA runtime themselves.  The reference's callers
 * free those results with cudaFree (testers/pst-tester-functions.tu:711-713). */
pst_status pst_free(void *ptr_d);

/* ------------------------------------------------------------------------- */
/* Tree                                                                       */

/* Device bytes needed to build and hold a tree of n points, including the
 * construction working set.  Replaces StaticPSTGPU::calcGlobalMemNeeded
 * (pst/static-pst-gpu.h:132, pst/static-pst-gpu.tu:648-671). */
pst_status pst_mem_needed(pst_dtype dtype, pst_idtype idtype, uint64_t n, uint64_t *bytes);

/* Builds a tree from n PointStruct records in device memory.  The input is only
 * read; the tree keeps its own copy of the values.  Returns after construction
 * has completed.  n == 0 gives an empty tree.  Replaces the StaticPSTGPU
 * constructor (pst/static-pst-gpu.h:76-78, pst/static-pst-gpu.tu:21-437) and the
 * StaticPSTGPUArr constructor (pst/static-pst-gpu-arr.h:51-54). */
pst_status pst_create(pst_tree **out, pst_dtype dtype, pst_idtype idtype, const void *pts_d,
                      uint64_t n, pst_stream_t stream);

/* Frees the tree.  Replaces ~StaticPSTGPU (pst/static-pst-gpu.h:80-88). */
pst_status pst_destroy(pst_tree *tree);

/* Tree images (no reference counterpart: the reference rebuilds every tree from
 * its points).  An image is a 64-byte header followed by the tree's device
 * arrays; loading one recreates the tree on the current device without a build.
 * pst_image_size gives the bytes pst_save writes; pst_save copies the image to
 * host memory of `capacity` bytes (PST_ERR_CAPACITY if too small; *written = the
 * image size either way); pst_load creates a tree from an image in host memory
 * (PST_ERR_INVALID for a bad or truncated image, PST_ERR_UNSUPPORTED for another
 * image version).  The _file forms stream the image through pinned staging
 * buffers, the disk transfer overlapping the host-device copy. */
pst_status pst_image_size(const pst_tree *tree, uint64_t *bytes);
pst_status pst_save(const pst_tree *tree, void *host, uint64_t capacity, uint64_t *written,
                    pst_stream_t stream);
pst_status pst_load(pst_tree **out, const void *host, uint64_t size, pst_stream_t stream);
pst_status pst_save_file(const pst_tree *tree, const char *path);
pst_status pst_load_file(pst_tree **out, const char *path, pst_stream_t stream);

/* Tree facts: number of points, levels, slots of the reference's layout
 * (2^levels - 1), device bytes held.  Any output pointer may be NULL.
 * Replaces the getters of pst/static-pst-gpu.h:96-98 and the slot count of
 * pst/static-pst-gpu.h:345-353. */
pst_status pst_info(const pst_tree *tree, uint64_t *n, uint32_t *levels, uint64_t *slots,
                    uint64_t *device_bytes, pst_dtype *dtype, pst_idtype *idtype);

/* Copies the tree to host buffers in the reference's field layout (slot s = heap
 * index with the root at 0; each array holds `slots` entries; ids may be NULL for
 * an id-less tree).  Unused slots are zero, as in the reference's value-initialised
 * allocation.  This is the data StaticPSTGPU::print walks
 * (pst/static-pst-gpu.h:93, pst/static-pst-gpu.tu:440-483). */
pst_status pst_export(const pst_tree *tree, void *dim1, void *dim2, void *med, uint32_t *ids,
                      uint8_t *bitcodes);

/* One query, drop-in mode: allocates the result (exactly *count records, from the
 * library's stream-ordered result pool; the caller frees it with cudaFree as the
 * reference's callers do, or with cudaFreeAsync on a stream to avoid the
 * device-wide synchronisation cudaFree may take), blocks until the result is
 * complete, and sets *out_d = NULL, *count = 0 for an empty tree or an empty
 * result.  Replaces StaticPSTGPU::threeSidedSearch / twoSidedLeftSearch /
 * twoSidedRightSearch (pst/static-pst-gpu.h:103-128, pst/static-pst-gpu.tu:496-642)
 * and StaticPSTGPUArr::twoSidedLeftSearch (pst/static-pst-gpu-arr.h:85-91). */
pst_status pst_search(pst_tree *tree, const pst_query *query, pst_ret ret, void **out_d,
                      uint64_t *count, pst_stream_t stream);

/* Size prepass: the number of records the query would return (what the
 * reference's searches leave in num_res_elems, pst/static-pst-gpu.tu:533-538),
 * without producing them.  Blocks. */
pst_status pst_count(pst_tree *tree, const pst_query *query, uint64_t *count, pst_stream_t stream);

/* The three reference search calls with the reference's bound order. */
pst_status pst_three_sided(pst_tree *tree, pst_value min1, pst_value max1, pst_value min2,
                           pst_ret ret, void **out_d, uint64_t *count, pst_stream_t stream);
pst_status pst_two_sided_left(pst_tree *tree, pst_value max1, pst_value min2, pst_ret ret,
                              void **out_d, uint64_t *count, pst_stream_t stream);
pst_status pst_two_sided_right(pst_tree *tree, pst_value min1, pst_value min2, pst_ret ret,
                               void **out_d, uint64_t *count, pst_stream_t stream);

/* One query into a caller buffer of `capacity` records.  *count always receives
 * the full result size; PST_ERR_CAPACITY (nothing written) when it exceeds
 * capacity.  Blocks until complete.  No reference counterpart takes a caller
 * buffer; this is the search of pst/static-pst-gpu.tu:548-591 without its
 * per-call cudaMalloc. */
pst_status pst_search_into(pst_tree *tree, const pst_query *query, pst_ret ret, void *out_d,
                           uint64_t capacity, uint64_t *count, pst_stream_t stream);

/* One query into a caller buffer without allocating anything.  It has no
 * counterpart in the reference.  It is for callers that cannot allocate device
 * memory while they search: code whose device memory is all held by its own
 * allocator, and latency-critical loops that cannot take the device-wide
 * synchronisation of cudaMalloc/cudaFree.  Its working memory is a static 8 MiB
 * device array in the library (held by every GPU that loads it until the process
 * exits), which bounds the tree: at most 2^22 - 1 = 4,194,303 points, larger trees
 * are rejected with PST_ERR_CAPACITY before any work.  The tree must live on the
 * current device (PST_ERR_INVALID otherwise).  The result contract is
 * pst_search_into's: *count is the full size, PST_ERR_CAPACITY (nothing written)
 * when it exceeds `capacity`.  Blocks until complete.  The first call on a device
 * (and the first after a cudaDeviceReset) looks up the array's device address;
 * make that first call before any stream capture begins.  All calls on a device
 * share the array, so calls whose GPU work overlapped would race; calls from one
 * process are serialised (each holds a lock until its work has completed, also
 * when it fails). */
pst_status pst_search_noalloc(pst_tree *tree, const pst_query *query, pst_ret ret, void *out_d,
                              uint64_t capacity, uint64_t *count, pst_stream_t stream);

/* ------------------------------------------------------------------------- */
/* Batched queries: many queries of mixed kinds in one level-synchronous pass
 * (count prepass, exact offsets, emit), replayed from a captured CUDA graph.
 * Waiting calls with at most 32 queries start with a one-CTA pass over the upper
 * levels and launch per-level kernels only below where it stopped.
 * The reference has one query per launch (pst/static-pst-gpu.tu:496-642); this
 * is the batched form of the same searches. */

/* Launch shape of an engine.  The zero values are the library's defaults; the
 * project's autotuner (static-priority-search-tree_b200/autotune.py) times the
 * choices on the caller's own queries and caches the fastest per tree shape and
 * batch size (the reference launches one block of warp_multiplier x 32 threads per
 * query, pst/static-pst-gpu.tu:525-529). */
typedef struct pst_batch_opts {
	uint32_t max_queries;      /* capacity of the query buffer */
	uint64_t task_capacity;    /* initial frontier capacity in 64-slot block records (0 = auto) */
	uint32_t block_threads;    /* CTA size of the level and emit kernels: 128, 256 or 512 (0 = 256) */
	uint32_t blocks_per_sm;    /* level-kernel CTAs per SM (0 = as many as fit) */
	int32_t use_graph;         /* replay the pass from a captured CUDA graph */
	uint32_t emit_records;     /* records in flight per warp when ids are emitted: 4, 8 or 16 (0 = 8) */
	uint32_t top_pass_queries; /* largest waiting batch that starts with the one-CTA top pass, at
	                              most 1024 (0 = 32) */
} pst_batch_opts;

pst_status pst_batch_create(pst_batch **out, pst_tree *tree, const pst_batch_opts *opts);
pst_status pst_batch_destroy(pst_batch *batch);

/* Runs nq queries (host or device array of pst_query).  Results of query i are
 * records [offsets[i], offsets[i+1]) of out_d; offsets_d receives nq + 1 uint64
 * values (device memory).  *total (host) receives the number of records.  When
 * the result exceeds out_capacity records, nothing is written to out_d,
 * offsets are still valid and PST_ERR_CAPACITY is returned.  sync = 0 makes the
 * call asynchronous on `stream` (then *total is only valid after a stream sync
 * and capacity overflow is reported by pst_batch_status). */
pst_status pst_batch_run(pst_batch *batch, const pst_query *queries, uint32_t nq, int queries_on_device,
                         pst_ret ret, void *out_d, uint64_t out_capacity, uint64_t *offsets_d,
                         uint64_t *total, int sync, pst_stream_t stream);

/* Count prepass only: per-query result sizes into counts_d (nq uint64 values,
 * device memory; may be NULL).  Blocks until complete. */
pst_status pst_batch_count(pst_batch *batch, const pst_query *queries, uint32_t nq, int queries_on_device,
                           uint64_t *counts_d, uint64_t *total, pst_stream_t stream);

/* After an asynchronous run: PST_OK, PST_ERR_CAPACITY or PST_ERR_INTERNAL. */
pst_status pst_batch_status(pst_batch *batch, uint64_t *total);

/* Frontier statistics of the last synchronised pass (for profiling and byte
 * accounting): alive 32-slot chunk records over all levels, report-above seeds,
 * reported boundary nodes, points reported, and the records per level (up to 40
 * entries written to per_level when it is non-null). */
typedef struct pst_batch_stats {
	uint64_t records, seeds, boundary, points;
	uint32_t levels;
} pst_batch_stats;
pst_status pst_batch_last_stats(pst_batch *batch, pst_batch_stats *stats, uint32_t *per_level);

/* The engine's launch shape as resolved on its device: CTA size, level-kernel CTAs
 * per SM and grid, emit records in flight, top-pass batch limit (any pointer may be
 * NULL).  No reference counterpart (its launch shape is fixed per call,
 * pst/static-pst-gpu.tu:525-529). */
pst_status pst_batch_launch_shape(pst_batch *batch, uint32_t *block_threads, uint32_t *blocks_per_sm,
                                  uint32_t *grid, uint32_t *emit_records, uint32_t *top_pass_queries);

/* ------------------------------------------------------------------------- */
/* Serving: a request loop over several resident trees with continuous batching.
 * Requests that arrive while other batches are on the device join the next free
 * batch slot; each batch runs its count pass, and its emit is admitted when the
 * exact output bytes that pass predicts fit the free result arena.  Batches of
 * different trees and slots run on separate streams and overlap on the device.
 * Latency is measured from each request's arrival time to the moment its result
 * is in host memory.  One worker thread per server drives every batch: while
 * any batch is on the device it polls their events without sleeping (one CPU
 * core busy), and with nothing in flight it sleeps until a submission.  The
 * reference has no serving layer; each request is the search of
 * pst/static-pst-gpu.tu:496-642. */

typedef struct pst_server pst_server;

typedef struct pst_server_opts {
	uint32_t max_batch;        /* queries per batch (0 = 1024) */
	uint32_t slots_per_tree;   /* batches in flight per tree (0 = 2) */
	uint64_t out_budget_bytes; /* device bytes for results in flight (0 = 1 GiB) */
	int32_t use_graph;         /* replay each slot's pass from a CUDA graph */
	int32_t keep_results;      /* 1: results copied to host and kept for pst_server_take;
	                              2: copied to host (latency includes it) then dropped;
	                              0: results stay in device memory, only counts are kept */
	uint64_t hbm_headroom_bytes; /* 0: a batch waits until its results fit the arena (a batch
	                                larger than the arena is split, a request larger than it
	                                fails with PST_ERR_NOMEM); > 0: a batch that does not fit
	                                the arena is admitted into a device buffer of its own when
	                                free HBM (cudaMemGetInfo) stays above this many bytes with
	                                it, one such batch at a time */
} pst_server_opts;

typedef struct pst_server_stats {
	uint64_t submitted, completed, failed, cancelled, batches, points;
	uint64_t peak_out_bytes;   /* largest arena use seen */
	uint64_t spilled;          /* batches admitted into free HBM beyond the arena */
	double p50_ms, p90_ms, p99_ms, mean_ms, max_ms; /* over requests completed since the last reset */
	double busy_s;             /* wall time from the first arrival to the last completion */
	double worker_cpu_s;       /* CPU time of the server's worker thread since the last reset */
} pst_server_stats;

pst_status pst_server_create(pst_server **out, const pst_server_opts *opts);
/* Registers a resident tree (it must outlive the server); returns its index. */
pst_status pst_server_add_tree(pst_server *srv, pst_tree *tree, uint32_t *tree_index);
/* The same with the launch shape of the tree's batch engines taken from `tuning`
 * (block_threads, blocks_per_sm, emit_records, top_pass_queries; its other fields
 * are ignored: the server's opts set the batch size and graph replay), e.g. the
 * autotuner's choice for the tree (NULL = the defaults). */
pst_status pst_server_add_tree_tuned(pst_server *srv, pst_tree *tree, const pst_batch_opts *tuning,
                                     uint32_t *tree_index);
/* Queues n requests.  arrival_ns (CLOCK_MONOTONIC, may be NULL = now) is the
 * arrival time latency is measured from.  ids receives request ids. */
pst_status pst_server_submit(pst_server *srv, uint32_t n, const uint32_t *tree_index, const pst_query *queries,
                             pst_ret ret, const uint64_t *arrival_ns, uint64_t *ids);
/* Waits (bounded by timeout_ms) until request id is done; PST_ERR_TIMEOUT otherwise.
 * *status receives the request's own status, *count its result size. */
pst_status pst_server_wait(pst_server *srv, uint64_t id, uint32_t timeout_ms, pst_status *status, uint64_t *count);
/* Copies a finished request's result (kept results only) to host memory of
 * `capacity` records and forgets the request. */
pst_status pst_server_take(pst_server *srv, uint64_t id, void *host_out, uint64_t capacity, uint64_t *count);
/* Cancels a request that has not completed; its result is dropped. */
pst_status pst_server_cancel(pst_server *srv, uint64_t id);
/* Waits (bounded) until every submitted request is done. */
pst_status pst_server_drain(pst_server *srv, uint32_t timeout_ms);
pst_status pst_server_get_stats(pst_server *srv, pst_server_stats *stats);
pst_status pst_server_reset_stats(pst_server *srv);
pst_status pst_server_destroy(pst_server *srv);

/* ------------------------------------------------------------------------- */
/* Interval parallel search: every point with dim1 <= v <= dim2, by a full scan.
 * Drop-in mode: like the reference, the result buffer has room for all n points
 * (allocated from the library's result pool; the caller frees it with cudaFree)
 * and *count records are valid; it is
 * NULL for n == 0.  Blocks until complete.
 * Replaces intervalParallelSearch (interval-parallel-search/interval-parallel-search.h:29-66);
 * num_blocks is a launch hint (0 = automatic), threads_per_block is ignored. */
pst_status pst_ips_search(pst_dtype dtype, pst_idtype idtype, const void *pts_d, uint64_t n,
                          pst_value v, pst_ret ret, void **out_d, uint64_t *count,
                          uint32_t num_blocks, uint32_t threads_per_block, pst_stream_t stream);

/* Same scan into a caller buffer of `capacity` records (PST_ERR_CAPACITY when the
 * result is larger; *count is the full size either way). */
pst_status pst_ips_search_into(pst_dtype dtype, pst_idtype idtype, const void *pts_d, uint64_t n,
                               pst_value v, pst_ret ret, void *out_d, uint64_t capacity,
                               uint64_t *count, pst_stream_t stream);

/* ------------------------------------------------------------------------- */
/* Metacell formation over a scalar vertex volume (x fastest, then y, then z).  */

/* Metacell grid dims and count: ceil((pt_dims[i] - 1) / mc_dims[i]) per axis.
 * Replaces calcNumMetacells (helpers/isosurface-data-processing.h:23-36). */
pst_status pst_num_metacells(const uint32_t pt_dims[3], const uint32_t mc_dims[3],
                             uint32_t mc_grid[3], uint64_t *n_metacells);

/* Writes one PointStruct (min vertex value, max vertex value[, id]) per metacell,
 * at index id = mx + (my + mz*My)*Mx, into out_d (device, n_metacells records).
 * A metacell covers the vertices [m*mc, min(m*mc + mc, P - 1)] of each axis.
 * Replaces formMetacellTags (helpers/isosurface-data-processing.h:69-137) and,
 * with mc_dims = {1,1,1}, formVoxelTags (:140-203). */
pst_status pst_form_metacells(pst_dtype dtype, pst_idtype idtype, const void *vert_d,
                              const uint32_t pt_dims[3], const uint32_t mc_dims[3], void *out_d,
                              pst_stream_t stream);

/* ------------------------------------------------------------------------- */
/* Marching cubes over active metacells (float32 volumes), headless.            */

/* Triangles of the cells (voxel cubes) of the metacells ids_d[0..n_ids) (ids as
 * pst_form_metacells numbers them, e.g. the result of pst_two_sided_left(iso, iso)
 * on the metacell tree): a corner is inside when its value is >= iso; each
 * triangle is 9 floats (three vertices x, y, z in vertex-index units), wound so
 * that its normal points from inside to outside; output ordered by the given ids,
 * then cell (x fastest), then table order.  The triangle table is this library's
 * own (pst_mc_tables returns it: ntri[256], edges[256][15] with edge 4a + u + 2v
 * along axis a), giving a closed, consistently oriented surface.  No reference
 * counterpart runs headless: the reference's isosurface sample
 * (.marching-cubes/marchingCubes_kernel.cu:155-413) renders through OpenGL.
 * pst_mc_count returns the number of triangles; pst_mc_triangles writes them
 * into tri_d (capacity triangles; PST_ERR_CAPACITY with the full count otherwise). */
pst_status pst_mc_tables(uint8_t ntri[256], uint8_t edges[256 * 15]);
pst_status pst_mc_count(const float *vol_d, const uint32_t pt_dims[3], const uint32_t mc_dims[3],
                        const uint32_t *ids_d, uint64_t n_ids, float iso, uint64_t *n_triangles,
                        pst_stream_t stream);
pst_status pst_mc_triangles(const float *vol_d, const uint32_t pt_dims[3], const uint32_t mc_dims[3],
                            const uint32_t *ids_d, uint64_t n_ids, float iso, float *tri_d,
                            uint64_t capacity, uint64_t *n_triangles, pst_stream_t stream);

/* Reads a raw volume file (num_vertices values of dtype, x fastest, no header)
 * into device memory vert_d.  Replaces readInVertices
 * (helpers/isosurface-data-processing.h:205-229), which reads into host memory and
 * exits on a missing or short file; here those are PST_ERR_INVALID.  The file
 * streams through pinned double buffers: the disk read of one chunk overlaps the
 * host-to-device copy of the previous one. */
pst_status pst_read_volume(const char *path, pst_dtype dtype, uint64_t num_vertices, void *vert_d,
                           pst_stream_t stream);

/* readInVertices followed by formMetacellTags without holding the volume on the
 * device: the volume streams in z-slabs of metacell layers (about slab_bytes each;
 * 0 = 64 MiB), each slab reduced to its metacells while the next is read.  Output as
 * pst_form_metacells; the records are bit-identical to pst_form_metacells over the
 * whole volume. */
pst_status pst_form_metacells_from_file(const char *path, pst_dtype dtype, pst_idtype idtype,
                                        const uint32_t pt_dims[3], const uint32_t mc_dims[3], void *out_d,
                                        uint64_t slab_bytes, pst_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* PST_C_H */
