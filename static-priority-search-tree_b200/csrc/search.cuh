// Batched / single-query search engine (host side).
#pragma once

#include "tree.cuh"

namespace pst {

constexpr int BFS_THREADS = 256;
// Batches of at most this many queries (by default; pst_batch_opts.top_pass_queries
// sets it per engine, up to MAX_TOP_PASS_Q) start with the one-CTA top pass, which
// walks the upper levels without a kernel boundary between them.
constexpr uint32_t SMALL_BATCH_Q = 32;
constexpr uint32_t MAX_TOP_PASS_Q = 1024;

enum : uint32_t {
	BATCH_FLAG_TASK_OVERFLOW = 1u,  // frontier buffer too small (results incomplete)
	BATCH_FLAG_OUT_OVERFLOW = 2u,   // output buffer too small (nothing written)
	BATCH_FLAG_BAD_QUERY = 4u,      // a query kind out of range
	BATCH_FLAG_INTERNAL = 8u,       // a device-side consistency check failed
};

// Device control block of one pass; the host uploads a zeroed copy (with nq set)
// at the start of every pass.
struct BatchCtl {
	uint32_t lvl_cnt[40];   // alive records appended per level region
	uint32_t path_cnt[40];  // boundary-path tasks per level
	uint32_t seed_cnt[40];  // report-above seeds per level
	uint32_t rec_cnt;       // reported boundary nodes
	uint32_t nq;
	uint32_t flags;
	uint32_t cta_levels;    // levels already done by the one-CTA top pass (small batches)
	uint64_t need_tasks;
	uint64_t total;
	// start of each level region (the sum of the counts before it), written by the
	// kernel that fills the region, so the next kernel reads its bounds in one load
	// each instead of summing every count before them
	uint64_t lvl_base[40];
};

struct Batch {
	TreeStorage *tree = nullptr;
	uint32_t max_q = 0;
	bool use_graph = true;
	uint32_t threads = BFS_THREADS;  // CTA size of the level and emit kernels
	uint32_t emit_u = 8;             // records in flight per warp in the emit (ids)
	uint32_t top_q = SMALL_BATCH_Q;  // largest batch that starts with the one-CTA top pass
	uint32_t blocks_per_sm = 0;
	uint32_t grid = 0;
	// queries
	pst_query *q_raw = nullptr;
	pst_query *q_stage = nullptr;  // pinned staging for host query arrays
	uint32_t *kind = nullptr;
	void *min1 = nullptr, *max1 = nullptr, *min2 = nullptr;
	// frontier and results
	uint4 *rec = nullptr;       // alive records: (64-slot block base, query, reported-slot mask lo, hi)
	uint64_t task_cap = 0;      // alive-record capacity
	uint4 *path0 = nullptr, *path1 = nullptr;
	uint4 *seed0 = nullptr, *seed1 = nullptr;
	uint32_t path_cap = 0;
	uint4 *ro = nullptr;        // reported boundary nodes, as one-bit records
	uint32_t ro_cap = 0;
	uint64_t *counts = nullptr, *cursor = nullptr, *offsets = nullptr, *scan_tmp = nullptr;
	BatchCtl *ctl = nullptr;
	BatchCtl *ctl_host = nullptr;  // pinned, zeroed except nq
	const BatchCtl *ctl_host_d = nullptr;  // its device address (mapped pinned memory)
	BatchCtl last{};
	// captured passes, each for the stream it was captured for: the whole count pass,
	// and the top pass of small batches
	struct Graph {
		cudaGraphExec_t exec = nullptr;
		cudaStream_t stream = nullptr;
		void drop();
	};
	Graph full_graph, top_graph;

	~Batch();
	void init(TreeStorage *t, const pst_batch_opts &o);
	void release();
	void grow_tasks(uint64_t cap, cudaStream_t s);
	void stage_queries(const pst_query *q, uint32_t nq, bool on_device, cudaStream_t s);
	// Whole count pass (every level kernel and the scan), asynchronous.
	void launch_count(cudaStream_t s);
	// Top pass of a small batch (nq <= top_q), asynchronous: when it stops
	// above the bottom (ctl->cta_levels < tree levels), launch_count_rest finishes it.
	void launch_count_top(cudaStream_t s);
	void launch_count_rest(uint32_t from, cudaStream_t s);
	// Count pass with the host waiting for it: the top pass for small batches, the
	// whole pass otherwise; grows the frontier buffer until the pass fits.
	void count_sync(cudaStream_t s, uint64_t *total);
	void count_full_sync(cudaStream_t s, uint64_t *total);
	void count_small_sync(cudaStream_t s, uint64_t *total);
	void enqueue_counting(cudaStream_t s);
	void enqueue_counting_top(cudaStream_t s);
	void enqueue_emit(pst_ret ret, void *out, uint64_t capacity, cudaStream_t s);
	pst_status read_ctl(cudaStream_t s, uint64_t *total);
	uint64_t record_size(pst_ret ret) const;

  private:
	template <typename T>
	void enqueue_count(cudaStream_t s);
	template <typename T>
	void enqueue_count_top(cudaStream_t s);
	template <typename T>
	void enqueue_count_rest(uint32_t from, cudaStream_t s);
	void launch_graph(Graph &g, void (Batch::*enqueue)(cudaStream_t), cudaStream_t s);
	template <typename T>
	void enqueue_emit_v(pst_ret ret, void *out, uint64_t capacity, cudaStream_t s);
	template <typename T, bool HAS_ID, bool POINTS>
	void enqueue_emit_t(void *out, uint64_t capacity, cudaStream_t s);
};

// One query into a caller buffer using only the library's static device scratch
// (no allocation); see pst_search_noalloc in include/pst_c.h.
uint64_t search_noalloc(TreeStorage &t, const pst_query &q, pst_ret ret, void *out, uint64_t capacity, cudaStream_t s);

}  // namespace pst
