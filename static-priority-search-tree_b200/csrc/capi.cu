// C ABI (include/pst_c.h): argument checks, error translation, and the drop-in
// search semantics of the reference (callee-allocated results, blocking calls).
#include <cstdio>
#include <functional>
#include <memory>
#include <mutex>
#include <new>
#include <string>

#include "scan_kernels.cuh"
#include "search.cuh"
#include "tree.cuh"

struct pst_batch {
	pst::Batch b;
	pst_tree *tree;
};

namespace pst {

namespace {
thread_local std::string g_last_error;
}

void fail(pst_status st, const std::string &msg) { throw Error{st, msg}; }

void check_cuda(cudaError_t e, const char *what)
{
	if (e == cudaSuccess)
		return;
	cudaGetLastError();
	fail(e == cudaErrorMemoryAllocation ? PST_ERR_NOMEM : PST_ERR_CUDA,
	     std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

const DeviceInfo &device_info()
{
	static thread_local DeviceInfo cache[64];
	static thread_local bool have[64] = {};
	int dev = 0;
	check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
	if (dev < 0 || dev >= 64)
		fail(PST_ERR_CUDA, "device index out of range");
	if (!have[dev]) {
		DeviceInfo d{};
		d.device = dev;
		check_cuda(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
		int smem = 0;
		check_cuda(cudaDeviceGetAttribute(&smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev), "cudaDeviceGetAttribute");
		d.smem_optin = (size_t) smem;
		cache[dev] = d;
		have[dev] = true;
	}
	return cache[dev];
}

static void require_device()
{
	int n = 0;
	cudaError_t e = cudaGetDeviceCount(&n);
	if (e != cudaSuccess || n == 0) {
		cudaGetLastError();
		fail(PST_ERR_CUDA, std::string("no CUDA device available: ") + cudaGetErrorString(e));
	}
}

static void check_types(pst_dtype dt, pst_idtype it)
{
	if (point_size(dt, it) == 0)
		fail(PST_ERR_INVALID, "invalid dtype/idtype");
}

static pst_status translate(const std::exception_ptr &ep)
{
	try {
		std::rethrow_exception(ep);
	} catch (const Error &e) {
		g_last_error = e.msg;
		return e.status;
	} catch (const std::bad_alloc &) {
		g_last_error = "host allocation failed";
		return PST_ERR_NOMEM;
	} catch (const std::exception &e) {
		g_last_error = e.what();
		return PST_ERR_INTERNAL;
	} catch (...) {
		g_last_error = "unknown error";
		return PST_ERR_INTERNAL;
	}
}

template <typename F>
static pst_status guarded(F &&f)
{
	try {
		f();
		g_last_error.clear();
		return PST_OK;
	} catch (...) {
		return translate(std::current_exception());
	}
}

pst_status guarded_call(const std::function<void()> &f) { return guarded(f); }

// Results handed to the caller (the drop-in searches' cudaMalloc'd arrays) come
// from a stream-ordered pool per device that keeps up to RESULT_POOL_KEEP bytes of
// freed memory for reuse, instead of a cudaMalloc per call (which, with the
// caller's cudaFree, costs more than the search itself).  The caller still frees a
// result with cudaFree, which accepts pool memory and does not synchronise for it:
// the call has waited for every write to the result before returning.
constexpr uint64_t RESULT_POOL_KEEP = 1ull << 30;

static cudaMemPool_t result_pool()
{
	static std::mutex mu;
	static cudaMemPool_t pools[64] = {};
	const int dev = device_info().device;
	std::lock_guard<std::mutex> lk(mu);
	if (!pools[dev]) {
		cudaMemPoolProps p{};
		p.allocType = cudaMemAllocationTypePinned;
		p.location.type = cudaMemLocationTypeDevice;
		p.location.id = dev;
		cudaMemPool_t pool = nullptr;
		check_cuda(cudaMemPoolCreate(&pool, &p), "cudaMemPoolCreate(results)");
		uint64_t keep = RESULT_POOL_KEEP;
		check_cuda(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
		pools[dev] = pool;
	}
	return pools[dev];
}

static void malloc_result(void **out, uint64_t bytes, cudaStream_t s)
{
	cudaError_t e = cudaMallocFromPoolAsync(out, bytes, result_pool(), s);
	if (e != cudaSuccess) {
		*out = nullptr;
		if (e == cudaErrorMemoryAllocation) {
			cudaGetLastError();
			fail(PST_ERR_NOMEM, "result allocation of " + std::to_string(bytes) + " B failed");
		}
		check_cuda(e, "cudaMallocFromPoolAsync(result)");
	}
}

static Batch &single_engine(pst_tree *tr)
{
	if (!tr->t.single) {
		pst_batch_opts o{};
		o.max_queries = 1;
		o.use_graph = 1;
		auto *b = new Batch();
		try {
			b->init(&tr->t, o);
		} catch (...) {
			delete b;
			throw;
		}
		tr->t.single = b;
	}
	return *tr->t.single;
}

// One query; out_d either caller-owned (capacity) or allocated here (alloc = true).
static uint64_t run_single(pst_tree *tr, const pst_query *q, pst_ret ret, void **out_d, uint64_t capacity, bool alloc,
                           cudaStream_t s)
{
	if (!tr || !q)
		fail(PST_ERR_INVALID, "null tree or query");
	if (q->kind < PST_Q_THREE || q->kind > PST_Q_RIGHT)
		fail(PST_ERR_INVALID, "query kind must be PST_Q_THREE, PST_Q_LEFT or PST_Q_RIGHT");
	if (ret != PST_RET_IDS && ret != PST_RET_POINTS)
		fail(PST_ERR_INVALID, "bad return type");
	if (ret == PST_RET_IDS && tr->t.idtype != PST_ID_U32)
		fail(PST_ERR_UNSUPPORTED, "an id-less tree can only return points");
	if (alloc)
		*out_d = nullptr;
	if (tr->t.n == 0)
		return 0;
	std::lock_guard<std::mutex> lk(tr->t.mu);
	Batch &b = single_engine(tr);
	b.stage_queries(q, 1, false, s);
	uint64_t total = 0;
	b.count_sync(s, &total);
	if (total == 0)
		return 0;
	if (alloc) {
		malloc_result(out_d, total * b.record_size(ret), s);
	} else if (total > capacity) {
		return total;
	}
	b.enqueue_emit(ret, *out_d, alloc ? total : capacity, s);
	uint64_t t2 = 0;
	const pst_status st = b.read_ctl(s, &t2);
	if (st != PST_OK) {
		if (alloc) {
			cudaFreeAsync(*out_d, s);  // after whatever the stream still holds
			*out_d = nullptr;
		}
		fail(st, "search emit failed");
	}
	return total;
}

}  // namespace pst

using namespace pst;

extern "C" {

const char *pst_last_error(void) { return g_last_error.c_str(); }

const char *pst_version(void) { return "pst_b200 1.0 (sm_100a)"; }

size_t pst_point_size(pst_dtype dtype, pst_idtype idtype) { return point_size(dtype, idtype); }

pst_status pst_free(void *ptr_d)
{
	return guarded([&] {
		if (ptr_d)
			check_cuda(cudaFree(ptr_d), "cudaFree");
	});
}

pst_status pst_mem_needed(pst_dtype dtype, pst_idtype idtype, uint64_t n, uint64_t *bytes)
{
	return guarded([&] {
		check_types(dtype, idtype);
		if (!bytes)
			fail(PST_ERR_INVALID, "null output");
		*bytes = build_bytes_needed(dtype, idtype, n);
	});
}

pst_status pst_create(pst_tree **out, pst_dtype dtype, pst_idtype idtype, const void *pts_d, uint64_t n,
                      pst_stream_t stream)
{
	return guarded([&] {
		if (!out)
			fail(PST_ERR_INVALID, "null output handle");
		*out = nullptr;
		check_types(dtype, idtype);
		require_device();
		auto tr = std::make_unique<pst_tree>();
		tr->t.dtype = dtype;
		tr->t.idtype = idtype;
		check_cuda(cudaGetDevice(&tr->t.device), "cudaGetDevice");
		build_tree(tr->t, pts_d, n, reinterpret_cast<cudaStream_t>(stream));
		*out = tr.release();
	});
}

pst_status pst_image_size(const pst_tree *tree, uint64_t *bytes)
{
	return guarded([&] {
		if (!tree || !bytes)
			fail(PST_ERR_INVALID, "null argument");
		*bytes = serialized_size(tree->t);
	});
}

pst_status pst_save(const pst_tree *tree, void *host, uint64_t capacity, uint64_t *written, pst_stream_t stream)
{
	return guarded([&] {
		if (!tree)
			fail(PST_ERR_INVALID, "null tree");
		if (written)
			*written = serialized_size(tree->t);
		save_tree(tree->t, host, capacity, reinterpret_cast<cudaStream_t>(stream));
	});
}

pst_status pst_load(pst_tree **out, const void *host, uint64_t size, pst_stream_t stream)
{
	return guarded([&] {
		if (!out)
			fail(PST_ERR_INVALID, "null output handle");
		*out = nullptr;
		require_device();
		auto tr = std::make_unique<pst_tree>();
		check_cuda(cudaGetDevice(&tr->t.device), "cudaGetDevice");
		load_tree(tr->t, host, size, reinterpret_cast<cudaStream_t>(stream));
		*out = tr.release();
	});
}

pst_status pst_save_file(const pst_tree *tree, const char *path)
{
	return guarded([&] {
		if (!tree)
			fail(PST_ERR_INVALID, "null tree");
		save_tree_file(tree->t, path);
	});
}

pst_status pst_load_file(pst_tree **out, const char *path, pst_stream_t stream)
{
	return guarded([&] {
		if (!out)
			fail(PST_ERR_INVALID, "null output handle");
		*out = nullptr;
		require_device();
		auto tr = std::make_unique<pst_tree>();
		check_cuda(cudaGetDevice(&tr->t.device), "cudaGetDevice");
		load_tree_file(tr->t, path, reinterpret_cast<cudaStream_t>(stream));
		*out = tr.release();
	});
}

pst_status pst_destroy(pst_tree *tree)
{
	return guarded([&] {
		if (!tree)
			return;
		delete tree->t.single;
		tree->t.single = nullptr;
		free_tree(tree->t);
		delete tree;
	});
}

pst_status pst_info(const pst_tree *tree, uint64_t *n, uint32_t *levels, uint64_t *slots, uint64_t *device_bytes,
                    pst_dtype *dtype, pst_idtype *idtype)
{
	return guarded([&] {
		if (!tree)
			fail(PST_ERR_INVALID, "null tree");
		if (n)
			*n = tree->t.n;
		if (levels)
			*levels = tree->t.levels;
		if (slots)
			*slots = tree->t.levels ? (1ull << tree->t.levels) - 1 : 0;
		if (device_bytes)
			*device_bytes = tree->t.bytes;
		if (dtype)
			*dtype = tree->t.dtype;
		if (idtype)
			*idtype = tree->t.idtype;
	});
}

pst_status pst_export(const pst_tree *tree, void *dim1, void *dim2, void *med, uint32_t *ids, uint8_t *bitcodes)
{
	return guarded([&] {
		if (!tree)
			fail(PST_ERR_INVALID, "null tree");
		if (tree->t.n && (!dim1 || !dim2 || !med || !bitcodes || (tree->t.idtype == PST_ID_U32 && !ids)))
			fail(PST_ERR_INVALID, "null export buffer");
		export_tree(tree->t, dim1, dim2, med, tree->t.idtype == PST_ID_U32 ? ids : nullptr, bitcodes);
	});
}

pst_status pst_count(pst_tree *tree, const pst_query *query, uint64_t *count, pst_stream_t stream)
{
	return guarded([&] {
		if (!count)
			fail(PST_ERR_INVALID, "null output");
		*count = 0;
		void *none = nullptr;
		*count = run_single(tree, query, PST_RET_POINTS, &none, 0, false, reinterpret_cast<cudaStream_t>(stream));
	});
}

pst_status pst_search(pst_tree *tree, const pst_query *query, pst_ret ret, void **out_d, uint64_t *count,
                      pst_stream_t stream)
{
	return guarded([&] {
		if (!out_d || !count)
			fail(PST_ERR_INVALID, "null output");
		*count = 0;
		*count = run_single(tree, query, ret, out_d, 0, true, reinterpret_cast<cudaStream_t>(stream));
	});
}

pst_status pst_three_sided(pst_tree *tree, pst_value min1, pst_value max1, pst_value min2, pst_ret ret, void **out_d,
                           uint64_t *count, pst_stream_t stream)
{
	pst_query q{};
	q.kind = PST_Q_THREE;
	q.min1 = min1;
	q.max1 = max1;
	q.min2 = min2;
	return pst_search(tree, &q, ret, out_d, count, stream);
}

pst_status pst_two_sided_left(pst_tree *tree, pst_value max1, pst_value min2, pst_ret ret, void **out_d,
                              uint64_t *count, pst_stream_t stream)
{
	pst_query q{};
	q.kind = PST_Q_LEFT;
	q.max1 = max1;
	q.min2 = min2;
	return pst_search(tree, &q, ret, out_d, count, stream);
}

pst_status pst_two_sided_right(pst_tree *tree, pst_value min1, pst_value min2, pst_ret ret, void **out_d,
                               uint64_t *count, pst_stream_t stream)
{
	pst_query q{};
	q.kind = PST_Q_RIGHT;
	q.min1 = min1;
	q.min2 = min2;
	return pst_search(tree, &q, ret, out_d, count, stream);
}

pst_status pst_search_into(pst_tree *tree, const pst_query *query, pst_ret ret, void *out_d, uint64_t capacity,
                           uint64_t *count, pst_stream_t stream)
{
	uint64_t total = 0;
	pst_status st = guarded([&] {
		if (!count)
			fail(PST_ERR_INVALID, "null count");
		void *o = out_d;
		total = run_single(tree, query, ret, &o, capacity, false, reinterpret_cast<cudaStream_t>(stream));
		*count = total;
	});
	if (st == PST_OK && total > capacity) {
		g_last_error = "result of " + std::to_string(total) + " records exceeds capacity " + std::to_string(capacity);
		return PST_ERR_CAPACITY;
	}
	return st;
}

pst_status pst_search_noalloc(pst_tree *tree, const pst_query *query, pst_ret ret, void *out_d, uint64_t capacity,
                              uint64_t *count, pst_stream_t stream)
{
	uint64_t total = 0;
	pst_status st = guarded([&] {
		if (!tree || !query || !count)
			fail(PST_ERR_INVALID, "null tree, query or count");
		if (ret != PST_RET_IDS && ret != PST_RET_POINTS)
			fail(PST_ERR_INVALID, "bad return type");
		if (ret == PST_RET_IDS && tree->t.idtype != PST_ID_U32)
			fail(PST_ERR_UNSUPPORTED, "an id-less tree can only return points");
		*count = 0;
		if (tree->t.n == 0)
			return;
		if (!out_d && capacity)
			fail(PST_ERR_INVALID, "null output buffer");
		total = search_noalloc(tree->t, *query, ret, out_d, capacity, reinterpret_cast<cudaStream_t>(stream));
		*count = total;
	});
	if (st == PST_OK && total > capacity) {
		g_last_error = "result of " + std::to_string(total) + " records exceeds capacity " + std::to_string(capacity);
		return PST_ERR_CAPACITY;
	}
	return st;
}

pst_status pst_batch_create(pst_batch **out, pst_tree *tree, const pst_batch_opts *opts)
{
	return guarded([&] {
		if (!out || !tree)
			fail(PST_ERR_INVALID, "null argument");
		*out = nullptr;
		pst_batch_opts o{};
		if (opts)
			o = *opts;
		else
			o.use_graph = 1;
		if (o.max_queries == 0)
			fail(PST_ERR_INVALID, "max_queries must be positive");
		auto b = std::make_unique<pst_batch>();
		b->tree = tree;
		b->b.init(&tree->t, o);
		*out = b.release();
	});
}

pst_status pst_batch_destroy(pst_batch *batch)
{
	return guarded([&] { delete batch; });
}

pst_status pst_batch_run(pst_batch *batch, const pst_query *queries, uint32_t nq, int queries_on_device, pst_ret ret,
                         void *out_d, uint64_t out_capacity, uint64_t *offsets_d, uint64_t *total, int sync,
                         pst_stream_t stream)
{
	pst_status result = PST_OK;
	pst_status st = guarded([&] {
		if (!batch)
			fail(PST_ERR_INVALID, "null batch");
		Batch &b = batch->b;
		cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
		if (ret != PST_RET_IDS && ret != PST_RET_POINTS)
			fail(PST_ERR_INVALID, "bad return type");
		if (ret == PST_RET_IDS && b.tree->idtype != PST_ID_U32)
			fail(PST_ERR_UNSUPPORTED, "an id-less tree can only return points");
		b.stage_queries(queries, nq, queries_on_device != 0, s);
		uint64_t tot = 0;
		if (sync) {
			b.count_sync(s, &tot);
			if (offsets_d)
				check_cuda(cudaMemcpyAsync(offsets_d, b.offsets, ((size_t) nq + 1) * 8, cudaMemcpyDeviceToDevice, s),
				           "copy offsets");
			if (total)
				*total = tot;
			if (tot > out_capacity) {
				check_cuda(cudaStreamSynchronize(s), "sync");
				result = PST_ERR_CAPACITY;
				return;
			}
			if (tot)
				b.enqueue_emit(ret, out_d, out_capacity, s);
			result = b.read_ctl(s, nullptr);
		} else {
			b.launch_count(s);
			b.enqueue_emit(ret, out_d, out_capacity, s);
			if (offsets_d)
				check_cuda(cudaMemcpyAsync(offsets_d, b.offsets, ((size_t) nq + 1) * 8, cudaMemcpyDeviceToDevice, s),
				           "copy offsets");
			if (total)
				check_cuda(cudaMemcpyAsync(total, &b.ctl->total, 8, cudaMemcpyDeviceToHost, s), "copy total");
		}
	});
	if (st != PST_OK)
		return st;
	if (result != PST_OK)
		g_last_error = result == PST_ERR_CAPACITY ? "batch result exceeds out_capacity" : "batch pass failed";
	return result;
}

pst_status pst_batch_count(pst_batch *batch, const pst_query *queries, uint32_t nq, int queries_on_device,
                           uint64_t *counts_d, uint64_t *total, pst_stream_t stream)
{
	return guarded([&] {
		if (!batch)
			fail(PST_ERR_INVALID, "null batch");
		Batch &b = batch->b;
		cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
		b.stage_queries(queries, nq, queries_on_device != 0, s);
		uint64_t tot = 0;
		b.count_sync(s, &tot);
		if (counts_d && nq)
			check_cuda(cudaMemcpyAsync(counts_d, b.counts, (size_t) nq * 8, cudaMemcpyDeviceToDevice, s), "copy counts");
		check_cuda(cudaStreamSynchronize(s), "sync");
		if (total)
			*total = tot;
	});
}

pst_status pst_batch_status(pst_batch *batch, uint64_t *total)
{
	pst_status result = PST_OK;
	pst_status st = guarded([&] {
		if (!batch)
			fail(PST_ERR_INVALID, "null batch");
		result = batch->b.read_ctl(nullptr, total);
	});
	return st != PST_OK ? st : result;
}

pst_status pst_batch_last_stats(pst_batch *batch, pst_batch_stats *stats, uint32_t *per_level)
{
	return guarded([&] {
		if (!batch || !stats)
			fail(PST_ERR_INVALID, "null argument");
		const BatchCtl &c = batch->b.last;
		pst_batch_stats st{};
		st.levels = batch->b.tree->levels;
		for (uint32_t d = 0; d < 40; d++) {
			st.records += c.lvl_cnt[d];
			st.seeds += c.seed_cnt[d];
			if (per_level)
				per_level[d] = c.lvl_cnt[d];
		}
		st.boundary = c.rec_cnt;
		st.points = c.total;
		*stats = st;
	});
}

pst_status pst_batch_launch_shape(pst_batch *batch, uint32_t *block_threads, uint32_t *blocks_per_sm, uint32_t *grid,
                                  uint32_t *emit_records, uint32_t *top_pass_queries)
{
	return guarded([&] {
		if (!batch)
			fail(PST_ERR_INVALID, "null argument");
		const Batch &b = batch->b;
		if (block_threads)
			*block_threads = b.threads;
		if (blocks_per_sm)
			*blocks_per_sm = b.blocks_per_sm;
		if (grid)
			*grid = b.grid;
		if (emit_records)
			*emit_records = b.emit_u;
		if (top_pass_queries)
			*top_pass_queries = b.top_q;
	});
}

// The result counter of an interval search: one device word and one pinned host
// word per calling thread and device, made on first use and kept (a call waits for
// its count before it returns, so a thread's calls never overlap).
namespace {
struct IpsCounter {
	unsigned long long *dev = nullptr;
	unsigned long long *host = nullptr;
};
struct IpsCounters {
	IpsCounter c[64];
	~IpsCounters()
	{
		for (IpsCounter &x : c) {
			if (x.dev)
				cudaFree(x.dev);
			if (x.host)
				cudaFreeHost(x.host);
		}
	}
};
thread_local IpsCounters t_ips_counters;

IpsCounter &ips_counter()
{
	const int dev = device_info().device;
	IpsCounter &x = t_ips_counters.c[dev];
	if (!x.dev) {
		check_cuda(cudaMalloc((void **) &x.dev, 8), "cudaMalloc(interval search counter)");
		if (cudaMallocHost((void **) &x.host, 8) != cudaSuccess) {
			cudaGetLastError();
			cudaFree(x.dev);
			x.dev = nullptr;
			fail(PST_ERR_NOMEM, "pinned interval search counter");
		}
	}
	return x;
}
}  // namespace

static uint64_t ips_common(pst_dtype dtype, pst_idtype idtype, const void *pts_d, uint64_t n, pst_value v, pst_ret ret,
                           void *out, uint64_t cap, uint32_t blocks, cudaStream_t s)
{
	IpsCounter &ctr = ips_counter();
	check_cuda(cudaMemsetAsync(ctr.dev, 0, 8, s), "memset");
	ips_run(dtype, idtype, ret, pts_d, n, v, out, cap, ctr.dev, blocks, s);
	check_cuda(cudaMemcpyAsync(ctr.host, ctr.dev, 8, cudaMemcpyDeviceToHost, s), "copy count");
	check_cuda(cudaStreamSynchronize(s), "sync");
	return *ctr.host;
}

pst_status pst_ips_search(pst_dtype dtype, pst_idtype idtype, const void *pts_d, uint64_t n, pst_value v, pst_ret ret,
                          void **out_d, uint64_t *count, uint32_t num_blocks, uint32_t threads_per_block,
                          pst_stream_t stream)
{
	(void) threads_per_block;
	return guarded([&] {
		if (!out_d || !count)
			fail(PST_ERR_INVALID, "null output");
		check_types(dtype, idtype);
		*out_d = nullptr;
		*count = 0;
		if (n == 0)
			return;
		if (!pts_d)
			fail(PST_ERR_INVALID, "null point array");
		require_device();
		const uint64_t rs = ret == PST_RET_IDS ? 4 : point_size(dtype, idtype);
		// The reference allocates room for every point (interval-parallel-search.h:35).
		malloc_result(out_d, n * rs, reinterpret_cast<cudaStream_t>(stream));
		try {
			*count = ips_common(dtype, idtype, pts_d, n, v, ret, *out_d, n, num_blocks,
			                    reinterpret_cast<cudaStream_t>(stream));
		} catch (...) {
			cudaFreeAsync(*out_d, reinterpret_cast<cudaStream_t>(stream));  // after the stream's work
			*out_d = nullptr;
			throw;
		}
	});
}

pst_status pst_ips_search_into(pst_dtype dtype, pst_idtype idtype, const void *pts_d, uint64_t n, pst_value v,
                               pst_ret ret, void *out_d, uint64_t capacity, uint64_t *count, pst_stream_t stream)
{
	uint64_t c = 0;
	pst_status st = guarded([&] {
		if (!count)
			fail(PST_ERR_INVALID, "null count");
		check_types(dtype, idtype);
		*count = 0;
		if (n == 0)
			return;
		if (!pts_d)
			fail(PST_ERR_INVALID, "null point array");
		require_device();
		c = ips_common(dtype, idtype, pts_d, n, v, ret, out_d, capacity, 0, reinterpret_cast<cudaStream_t>(stream));
		*count = c;
	});
	if (st == PST_OK && c > capacity) {
		g_last_error = "interval search result exceeds capacity";
		return PST_ERR_CAPACITY;
	}
	return st;
}

pst_status pst_num_metacells(const uint32_t pt_dims[3], const uint32_t mc_dims[3], uint32_t mc_grid[3],
                             uint64_t *n_metacells)
{
	return guarded([&] {
		if (!pt_dims || !mc_dims)
			fail(PST_ERR_INVALID, "null dims");
		uint64_t n = 1;
		for (int i = 0; i < 3; i++) {
			if (mc_dims[i] == 0 || pt_dims[i] < 2)
				fail(PST_ERR_INVALID, "each vertex dim must be >= 2 and each metacell dim >= 1");
			const uint32_t m = (pt_dims[i] - 1) / mc_dims[i] + ((pt_dims[i] - 1) % mc_dims[i] ? 1 : 0);
			if (mc_grid)
				mc_grid[i] = m;
			n *= m;
		}
		if (n_metacells)
			*n_metacells = n;
	});
}

pst_status pst_form_metacells(pst_dtype dtype, pst_idtype idtype, const void *vert_d, const uint32_t pt_dims[3],
                              const uint32_t mc_dims[3], void *out_d, pst_stream_t stream)
{
	return guarded([&] {
		check_types(dtype, idtype);
		uint32_t M[3];
		uint64_t nm = 0;
		if (pst_num_metacells(pt_dims, mc_dims, M, &nm) != PST_OK)
			fail(PST_ERR_INVALID, g_last_error);
		if (nm >= (1ull << 32) && idtype == PST_ID_U32)
			fail(PST_ERR_INVALID, "metacell ids must fit in 32 bits");
		if (!vert_d || !out_d)
			fail(PST_ERR_INVALID, "null buffer");
		require_device();
		metacells_run(dtype, idtype, vert_d, pt_dims, mc_dims, M, out_d, reinterpret_cast<cudaStream_t>(stream));
	});
}

pst_status pst_read_volume(const char *path, pst_dtype dtype, uint64_t num_vertices, void *vert_d,
                           pst_stream_t stream)
{
	return guarded([&] {
		check_types(dtype, PST_ID_NONE);
		require_device();
		read_volume(path, dtype, num_vertices, vert_d, reinterpret_cast<cudaStream_t>(stream));
	});
}

pst_status pst_form_metacells_from_file(const char *path, pst_dtype dtype, pst_idtype idtype,
                                        const uint32_t pt_dims[3], const uint32_t mc_dims[3], void *out_d,
                                        uint64_t slab_bytes, pst_stream_t stream)
{
	return guarded([&] {
		check_types(dtype, idtype);
		uint32_t M[3];
		uint64_t nm = 0;
		if (pst_num_metacells(pt_dims, mc_dims, M, &nm) != PST_OK)
			fail(PST_ERR_INVALID, g_last_error);
		if (nm >= (1ull << 32) && idtype == PST_ID_U32)
			fail(PST_ERR_INVALID, "metacell ids must fit in 32 bits");
		require_device();
		metacells_from_file(path, dtype, idtype, pt_dims, mc_dims, M, out_d, slab_bytes,
		                    reinterpret_cast<cudaStream_t>(stream));
	});
}

pst_status pst_mc_tables(uint8_t ntri[256], uint8_t edges[256 * 15])
{
	return guarded([&] {
		if (!ntri || !edges)
			fail(PST_ERR_INVALID, "null table buffer");
		mc_tables(ntri, edges);
	});
}

static void mc_check(const float *vol_d, const uint32_t pt_dims[3], const uint32_t mc_dims[3], const uint32_t *ids_d,
                     uint64_t n_ids)
{
	if (!pt_dims || !mc_dims)
		fail(PST_ERR_INVALID, "null dims");
	for (int i = 0; i < 3; i++) {
		if (pt_dims[i] < 2)
			fail(PST_ERR_INVALID, "a volume needs at least 2 vertices per axis");
		if (mc_dims[i] == 0)
			fail(PST_ERR_INVALID, "metacell dims must be positive");
	}
	if (n_ids && (!vol_d || !ids_d))
		fail(PST_ERR_INVALID, "null buffer");
	require_device();
}

pst_status pst_mc_count(const float *vol_d, const uint32_t pt_dims[3], const uint32_t mc_dims[3], const uint32_t *ids_d,
                        uint64_t n_ids, float iso, uint64_t *n_triangles, pst_stream_t stream)
{
	return guarded([&] {
		if (!n_triangles)
			fail(PST_ERR_INVALID, "null output");
		*n_triangles = 0;
		mc_check(vol_d, pt_dims, mc_dims, ids_d, n_ids);
		*n_triangles = mc_run(vol_d, pt_dims, mc_dims, ids_d, n_ids, iso, nullptr, 0, false,
		                      reinterpret_cast<cudaStream_t>(stream));
	});
}

pst_status pst_mc_triangles(const float *vol_d, const uint32_t pt_dims[3], const uint32_t mc_dims[3],
                            const uint32_t *ids_d, uint64_t n_ids, float iso, float *tri_d, uint64_t capacity,
                            uint64_t *n_triangles, pst_stream_t stream)
{
	return guarded([&] {
		if (!n_triangles)
			fail(PST_ERR_INVALID, "null output");
		*n_triangles = 0;
		mc_check(vol_d, pt_dims, mc_dims, ids_d, n_ids);
		const uint64_t total = mc_run(vol_d, pt_dims, mc_dims, ids_d, n_ids, iso, tri_d, capacity, true,
		                              reinterpret_cast<cudaStream_t>(stream));
		*n_triangles = total;
		if (total > capacity)
			fail(PST_ERR_CAPACITY, "triangle buffer holds " + std::to_string(capacity) + " of " +
			                           std::to_string(total) + " triangles");
	});
}

}  // extern "C"
