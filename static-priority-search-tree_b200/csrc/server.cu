// Serving loop: several resident trees, continuous batching, admission by the
// exact output bytes of each batch's count pass, overlapping batches on separate
// streams, p50/p99 latency from arrival to host result.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include <time.h>

#include <functional>

#include "search.cuh"

namespace pst {

namespace {

uint64_t now_ns()
{
	timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return (uint64_t) ts.tv_sec * 1000000000ull + (uint64_t) ts.tv_nsec;
}

enum ReqState { REQ_PENDING, REQ_RUNNING, REQ_DONE };

struct Request {
	uint64_t id;
	uint32_t tree;
	pst_query q;
	pst_ret ret;
	uint64_t arrival_ns;
	uint64_t done_ns = 0;
	ReqState state = REQ_PENDING;
	pst_status status = PST_OK;
	bool cancelled = false;
	uint64_t count = 0;
	std::vector<unsigned char> result;
};

// First-fit allocator over one device allocation (offsets, 256-byte granules).  When
// results go to host memory, a pinned host buffer of the same size mirrors it: a
// batch's results are copied to the same offsets there, so staging never allocates
// while requests wait.
struct Arena {
	char *base = nullptr;
	unsigned char *host = nullptr;
	uint64_t size = 0, used = 0, peak = 0;
	std::map<uint64_t, uint64_t> free_;  // offset -> length

	void init(uint64_t bytes, bool host_mirror)
	{
		size = (bytes + 255) / 256 * 256;
		check_cuda(cudaMalloc(&base, size), "cudaMalloc(result arena)");
		if (host_mirror)
			check_cuda(cudaMallocHost((void **) &host, size), "cudaMallocHost(result staging)");
		free_[0] = size;
	}
	~Arena()
	{
		if (base)
			cudaFree(base);
		if (host)
			cudaFreeHost(host);
	}
	bool alloc(uint64_t bytes, uint64_t *off)
	{
		bytes = std::max<uint64_t>((bytes + 255) / 256 * 256, 256);
		for (auto it = free_.begin(); it != free_.end(); ++it) {
			if (it->second >= bytes) {
				*off = it->first;
				const uint64_t rest = it->second - bytes, roff = it->first + bytes;
				free_.erase(it);
				if (rest)
					free_[roff] = rest;
				used += bytes;
				peak = std::max(peak, used);
				return true;
			}
		}
		return false;
	}
	void release(uint64_t off, uint64_t bytes)
	{
		bytes = std::max<uint64_t>((bytes + 255) / 256 * 256, 256);
		used -= bytes;
		auto it = free_.emplace(off, bytes).first;
		auto nx = std::next(it);
		if (nx != free_.end() && it->first + it->second == nx->first) {
			it->second += nx->second;
			free_.erase(nx);
		}
		if (it != free_.begin()) {
			auto pv = std::prev(it);
			if (pv->first + pv->second == it->first) {
				pv->second += it->second;
				free_.erase(it);
			}
		}
	}
};

// A small batch counts in two steps: its top pass (SLOT_TOP), then, only when that
// stopped above the bottom of the tree, the per-level kernels for the rest.
enum SlotPhase { SLOT_IDLE, SLOT_TOP, SLOT_COUNTING, SLOT_EMITTING };

struct Slot {
	Batch eng;
	cudaStream_t stream = nullptr;
	cudaEvent_t ev = nullptr;
	SlotPhase phase = SLOT_IDLE;
	std::vector<Request *> reqs;
	pst_ret ret = PST_RET_IDS;
	std::vector<pst_query> qhost;
	BatchCtl *ctl_h = nullptr;
	uint64_t *counts_h = nullptr;
	uint64_t *offs_h = nullptr;
	uint64_t out_off = 0, out_bytes = 0;
	uint64_t total = 0;
	bool spilled = false;        // results in a buffer of their own, outside the arena
	char *spill_d = nullptr;     // that buffer (stream-ordered allocation on the slot's stream)
	char *out_d = nullptr;       // where the emit writes this batch's results
	unsigned char *out_h = nullptr;  // and where they are staged in host memory (kept results)

	~Slot()
	{
		if (ev)
			cudaEventDestroy(ev);
		if (stream)
			cudaStreamDestroy(stream);
		if (ctl_h)
			cudaFreeHost(ctl_h);
		if (counts_h)
			cudaFreeHost(counts_h);
		if (offs_h)
			cudaFreeHost(offs_h);
	}
};

struct TreeSlots {
	TreeStorage *tree;
	uint32_t batch_limit = 1;       // halves when a batch's results cannot fit the arena
	std::deque<Request *> pending;  // worker-owned
	std::vector<std::unique_ptr<Slot>> slots;
};

}  // namespace

struct Server {
	pst_server_opts opts{};
	int device = 0;
	std::vector<std::unique_ptr<TreeSlots>> trees;
	Arena arena;
	// Batches whose results do not fit the arena may take a device buffer of their own
	// when free HBM allows (opts.hbm_headroom_bytes > 0), one such batch at a time;
	// its host staging buffer is kept and grown as needed.
	bool spill_busy = false;
	unsigned char *spill_h = nullptr;
	uint64_t spill_h_size = 0;
	std::mutex mu;
	std::condition_variable cv_work, cv_done;
	std::deque<Request *> inbox;
	std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
	uint64_t next_id = 1;
	uint64_t outstanding = 0;  // submitted and not yet done
	bool stop = false;
	std::thread worker;
	std::string worker_error;
	std::atomic<uint64_t> worker_cpu_ns{0};  // the worker thread's CPU time so far
	uint64_t worker_cpu_base = 0;            // ... at the last statistics reset
	// statistics (guarded by mu)
	pst_server_stats st{};
	std::vector<double> lat_ms;
	uint64_t first_arrival = 0, last_done = 0;

	void start()
	{
		worker = std::thread([this] { run(); });
	}

	void finish(Request *r, pst_status status, uint64_t count, std::vector<unsigned char> &&res)
	{
		std::lock_guard<std::mutex> lk(mu);
		r->done_ns = now_ns();
		r->status = status;
		r->count = count;
		r->result = std::move(res);
		r->state = REQ_DONE;
		outstanding--;
		if (r->cancelled) {
			st.cancelled++;
			r->result.clear();
		} else if (status == PST_OK) {
			st.completed++;
			st.points += count;
			lat_ms.push_back((double) (r->done_ns - r->arrival_ns) / 1e6);
			if (!first_arrival || r->arrival_ns < first_arrival)
				first_arrival = r->arrival_ns;
			last_done = std::max(last_done, r->done_ns);
		} else {
			st.failed++;
		}
	}

	// Whether free HBM, less the headroom, would hold `bytes` of results.
	bool could_spill(uint64_t bytes)
	{
		if (!opts.hbm_headroom_bytes)
			return false;
		size_t fr = 0, tot = 0;
		if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
			cudaGetLastError();
			return false;
		}
		return bytes + opts.hbm_headroom_bytes <= fr;
	}

	// Admits a batch whose results did not fit the arena into a device buffer of its
	// own, if no other batch holds one and free HBM (cudaMemGetInfo) stays above the
	// headroom with it.  The buffer is allocated on the slot's stream, so the
	// allocation waits for nothing on the device's other streams.
	bool try_spill(Slot &sl)
	{
		if (spill_busy || !could_spill(sl.out_bytes))
			return false;
		void *p = nullptr;
		if (cudaMallocAsync(&p, std::max<uint64_t>(sl.out_bytes, 256), sl.stream) != cudaSuccess) {
			cudaGetLastError();
			return false;
		}
		if (opts.keep_results && spill_h_size < sl.out_bytes) {
			if (spill_h)
				cudaFreeHost(spill_h);
			spill_h = nullptr;
			spill_h_size = 0;
			if (cudaMallocHost((void **) &spill_h, sl.out_bytes) != cudaSuccess) {
				cudaGetLastError();
				spill_h = nullptr;
				cudaFreeAsync(p, sl.stream);
				return false;
			}
			spill_h_size = sl.out_bytes;
		}
		sl.spill_d = static_cast<char *>(p);
		sl.out_d = sl.spill_d;
		sl.out_h = opts.keep_results ? spill_h : nullptr;
		spill_busy = true;
		std::lock_guard<std::mutex> lk(mu);
		st.spilled++;
		return true;
	}

	// Returns a finished batch's result space (arena range or spill buffer).
	void release_out(Slot &sl)
	{
		if (sl.spilled) {
			cudaFreeAsync(sl.spill_d, sl.stream);
			sl.spill_d = nullptr;
			sl.spilled = false;
			spill_busy = false;
		} else {
			arena.release(sl.out_off, sl.out_bytes);
		}
	}

	// One state-machine step of a slot; returns true if it made progress.
	bool step(TreeSlots &ts, Slot &sl)
	{
		if (sl.phase == SLOT_IDLE) {
			if (ts.pending.empty())
				return false;
			sl.reqs.clear();
			sl.qhost.clear();
			sl.ret = ts.pending.front()->ret;
			while (!ts.pending.empty() && sl.reqs.size() < ts.batch_limit && ts.pending.front()->ret == sl.ret) {
				Request *r = ts.pending.front();
				ts.pending.pop_front();
				bool skip;
				{
					std::lock_guard<std::mutex> lk(mu);
					skip = r->cancelled;
					if (!skip)
						r->state = REQ_RUNNING;
				}
				if (skip) {
					std::vector<unsigned char> none;
					finish(r, PST_OK, 0, std::move(none));
					continue;
				}
				sl.reqs.push_back(r);
				sl.qhost.push_back(r->q);
			}
			if (sl.reqs.empty())
				return true;
			launch_count(sl);
			return true;
		}
		if (cudaEventQuery(sl.ev) == cudaErrorNotReady)
			return false;
		check_cuda(cudaGetLastError(), "slot event");
		const uint32_t n = (uint32_t) sl.reqs.size();
		if (sl.phase == SLOT_TOP) {
			const BatchCtl &c = *sl.ctl_h;
			sl.phase = SLOT_COUNTING;
			if (!(c.flags & (BATCH_FLAG_TASK_OVERFLOW | BATCH_FLAG_BAD_QUERY | BATCH_FLAG_INTERNAL)) &&
			    c.cta_levels < sl.eng.tree->levels) {
				sl.eng.launch_count_rest(c.cta_levels, sl.stream);
				copy_count_results(sl, n);
				return true;
			}
			// the top pass reached the bottom (or failed): its results are final
		}
		if (sl.phase == SLOT_COUNTING) {
			const BatchCtl &c = *sl.ctl_h;
			if (c.flags & BATCH_FLAG_TASK_OVERFLOW) {
				// the pass stopped at the first level that overflowed, so deeper
				// levels will want more: grow generously
				sl.eng.grow_tasks(std::max<uint64_t>(c.need_tasks * 2, sl.eng.task_cap * 2), sl.stream);
				launch_count(sl);
				return true;
			}
			if (c.flags & (BATCH_FLAG_BAD_QUERY | BATCH_FLAG_INTERNAL)) {
				fail_all(sl, (c.flags & BATCH_FLAG_BAD_QUERY) ? PST_ERR_INVALID : PST_ERR_INTERNAL);
				return true;
			}
			const uint64_t rs = sl.eng.record_size(sl.ret);
			sl.total = c.total;
			if (sl.total == 0) {
				for (Request *r : sl.reqs) {
					std::vector<unsigned char> none;
					finish(r, PST_OK, 0, std::move(none));
				}
				sl.phase = SLOT_IDLE;
				notify_done();
				return true;
			}
			sl.out_bytes = sl.total * rs;
			sl.spilled = false;
			if (sl.out_bytes <= arena.size && arena.alloc(sl.out_bytes, &sl.out_off)) {
				sl.out_d = arena.base + sl.out_off;
				sl.out_h = arena.host ? arena.host + sl.out_off : nullptr;
			} else if (try_spill(sl)) {
				sl.spilled = true;
			} else if (sl.out_bytes <= arena.size || (spill_busy && could_spill(sl.out_bytes))) {
				return false;  // admitted once results in flight free the arena (or the spill)
			} else {
				// Requests that can never fit (neither the arena nor free HBM) fail; the
				// others go back to the queue front and the tree's batches shrink until
				// their results fit.
				ts.batch_limit = std::max<uint32_t>(1, n / 2);
				for (uint32_t i = n; i-- > 0;) {
					Request *r = sl.reqs[i];
					if (sl.counts_h[i] * rs > arena.size && !could_spill(sl.counts_h[i] * rs)) {
						std::vector<unsigned char> none;
						finish(r, PST_ERR_NOMEM, sl.counts_h[i], std::move(none));
					} else {
						std::lock_guard<std::mutex> lk(mu);
						r->state = REQ_PENDING;
						ts.pending.push_front(r);
					}
				}
				sl.phase = SLOT_IDLE;
				notify_done();
				return true;
			}
			sl.eng.enqueue_emit(sl.ret, sl.out_d, sl.total, sl.stream);
			check_cuda(cudaMemcpyAsync(sl.offs_h, sl.eng.offsets, ((size_t) n + 1) * 8, cudaMemcpyDeviceToHost,
			                           sl.stream), "copy offsets");
			if (opts.keep_results)
				check_cuda(cudaMemcpyAsync(sl.out_h, sl.out_d, sl.out_bytes, cudaMemcpyDeviceToHost, sl.stream),
				           "copy results");
			check_cuda(cudaMemcpyAsync(sl.ctl_h, sl.eng.ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, sl.stream),
			           "copy control");
			check_cuda(cudaEventRecord(sl.ev, sl.stream), "event");
			sl.phase = SLOT_EMITTING;
			{
				std::lock_guard<std::mutex> lk(mu);
				st.peak_out_bytes = std::max(st.peak_out_bytes, arena.peak);
			}
			return true;
		}
		// SLOT_EMITTING done
		if (sl.ctl_h->flags & (BATCH_FLAG_OUT_OVERFLOW | BATCH_FLAG_INTERNAL | BATCH_FLAG_TASK_OVERFLOW)) {
			release_out(sl);
			fail_all(sl, PST_ERR_INTERNAL);
			return true;
		}
		const uint64_t rs = sl.eng.record_size(sl.ret);
		const unsigned char *staged = sl.out_h;
		for (uint32_t i = 0; i < n; i++) {
			const uint64_t a = sl.offs_h[i], b = sl.offs_h[i + 1];
			std::vector<unsigned char> res;
			if (opts.keep_results == 1)
				res.assign(staged + a * rs, staged + b * rs);
			finish(sl.reqs[i], PST_OK, b - a, std::move(res));
		}
		release_out(sl);
		{
			std::lock_guard<std::mutex> lk(mu);
			st.batches++;
		}
		ts.batch_limit = std::min<uint32_t>(opts.max_batch, ts.batch_limit * 2);
		sl.phase = SLOT_IDLE;
		notify_done();
		return true;
	}

	void launch_count(Slot &sl)
	{
		const uint32_t n = (uint32_t) sl.reqs.size();
		sl.eng.stage_queries(sl.qhost.data(), n, false, sl.stream);
		if (n <= sl.eng.top_q) {
			sl.eng.launch_count_top(sl.stream);
			sl.phase = SLOT_TOP;
		} else {
			sl.eng.launch_count(sl.stream);
			sl.phase = SLOT_COUNTING;
		}
		copy_count_results(sl, n);
	}

	// Control block and per-query counts back to the slot's pinned buffers, then the
	// slot's event.
	void copy_count_results(Slot &sl, uint32_t n)
	{
		check_cuda(cudaMemcpyAsync(sl.ctl_h, sl.eng.ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, sl.stream),
		           "copy control");
		check_cuda(cudaMemcpyAsync(sl.counts_h, sl.eng.counts, (size_t) n * 8, cudaMemcpyDeviceToHost, sl.stream),
		           "copy counts");
		check_cuda(cudaEventRecord(sl.ev, sl.stream), "event");
	}

	void fail_all(Slot &sl, pst_status status)
	{
		for (Request *r : sl.reqs) {
			std::vector<unsigned char> none;
			finish(r, status, 0, std::move(none));
		}
		sl.phase = SLOT_IDLE;
		notify_done();
	}

	void notify_done() { cv_done.notify_all(); }

	void run()
	{
		try {
			check_cuda(cudaSetDevice(device), "cudaSetDevice");
			for (;;) {
				bool inflight = false;
				{
					std::unique_lock<std::mutex> lk(mu);
					while (!inbox.empty()) {
						Request *r = inbox.front();
						inbox.pop_front();
						trees[r->tree]->pending.push_back(r);
					}
					for (auto &ts : trees)
						for (auto &sl : ts->slots)
							inflight |= sl->phase != SLOT_IDLE;
					bool pending = false;
					for (auto &ts : trees)
						pending |= !ts->pending.empty();
					if (stop && !inflight && !pending)
						break;
				}
				bool progress = false;
				for (auto &ts : trees)
					for (auto &sl : ts->slots)
						progress |= step(*ts, *sl);
				{
					timespec c{};
					clock_gettime(CLOCK_THREAD_CPUTIME_ID, &c);
					worker_cpu_ns.store((uint64_t) c.tv_sec * 1000000000ull + (uint64_t) c.tv_nsec,
					                    std::memory_order_relaxed);
				}
				if (!progress) {
					if (inflight) {
						// GPU steps in flight: poll their events again right away.  A timed
						// wait here would add its whole sleep, rounded up by the OS timer
						// slack (about 100 us for a 20 us wait), to every step of every
						// request; a stream host function to wake this thread costs more
						// still, as it holds back the stream's next work.
						std::this_thread::yield();
					} else {
						std::unique_lock<std::mutex> lk(mu);
						if (inbox.empty() && !stop)
							cv_work.wait_for(lk, std::chrono::milliseconds(5));
					}
				}
			}
		} catch (const Error &e) {
			std::lock_guard<std::mutex> lk(mu);
			worker_error = e.msg;
		} catch (const std::exception &e) {
			std::lock_guard<std::mutex> lk(mu);
			worker_error = e.what();
		}
		cv_done.notify_all();
	}

	~Server()
	{
		{
			std::lock_guard<std::mutex> lk(mu);
			stop = true;
		}
		cv_work.notify_all();
		if (worker.joinable())
			worker.join();
		// the slots (and their streams) go with `trees` after this body; their spill
		// buffers were freed on their streams when their batches finished
		for (auto &ts : trees)
			for (auto &sl : ts->slots)
				if (sl->stream)
					cudaStreamSynchronize(sl->stream);
		if (spill_h)
			cudaFreeHost(spill_h);
	}
};

// ---------------------------------------------------------------------------
// C ABI glue (called from capi.cu).

Server *server_create(const pst_server_opts &o)
{
	auto s = std::make_unique<Server>();
	s->opts = o;
	if (!s->opts.max_batch)
		s->opts.max_batch = 1024;
	if (!s->opts.slots_per_tree)
		s->opts.slots_per_tree = 2;
	if (!s->opts.out_budget_bytes)
		s->opts.out_budget_bytes = 1ull << 30;
	check_cuda(cudaGetDevice(&s->device), "cudaGetDevice");
	s->arena.init(s->opts.out_budget_bytes, s->opts.keep_results != 0);
	s->start();
	return s.release();
}

uint32_t server_add_tree(Server *s, TreeStorage *t, const pst_batch_opts *tuning)
{
	if (t->device != s->device)
		fail(PST_ERR_INVALID, "all trees of a server must live on the server's device");
	auto ts = std::make_unique<TreeSlots>();
	ts->tree = t;
	ts->batch_limit = s->opts.max_batch;
	for (uint32_t i = 0; i < s->opts.slots_per_tree; i++) {
		auto sl = std::make_unique<Slot>();
		pst_batch_opts bo{};
		if (tuning) {
			// the tree's launch shape (the autotuner's choice); batch size and graph
			// replay stay the server's
			bo.block_threads = tuning->block_threads;
			bo.blocks_per_sm = tuning->blocks_per_sm;
			bo.emit_records = tuning->emit_records;
			bo.top_pass_queries = tuning->top_pass_queries;
		}
		bo.max_queries = s->opts.max_batch;
		bo.use_graph = s->opts.use_graph;
		// frontier sized from the tree (one 64-slot record per 8 points) so that batches
		// rarely grow it while requests wait
		bo.task_capacity = std::max<uint64_t>(1ull << 16, t->n / 8);
		sl->eng.init(t, bo);
		check_cuda(cudaStreamCreateWithFlags(&sl->stream, cudaStreamNonBlocking), "cudaStreamCreate");
		// warm-up passes: capture the slot's graphs (the whole count pass, and the top pass
		// of small batches) now rather than under the first requests
		{
			// an inverted 3-sided range walks one path and reports nothing
			pst_query q{};
			q.kind = PST_Q_THREE;
			if (t->dtype == PST_F32) {
				q.min1.f32 = 1.0f;
				q.max1.f32 = 0.0f;
			} else if (t->dtype == PST_F64) {
				q.min1.f64 = 1.0;
				q.max1.f64 = 0.0;
			} else {
				q.min1.i32 = 1;
				q.max1.i32 = 0;
			}
			sl->eng.stage_queries(&q, 1, false, sl->stream);
			uint64_t total = 0;
			sl->eng.count_full_sync(sl->stream, &total);
			sl->eng.count_small_sync(sl->stream, &total);
		}
		check_cuda(cudaEventCreateWithFlags(&sl->ev, cudaEventDisableTiming), "cudaEventCreate");
		check_cuda(cudaMallocHost((void **) &sl->ctl_h, sizeof(BatchCtl)), "cudaMallocHost");
		check_cuda(cudaMallocHost((void **) &sl->counts_h, (size_t) s->opts.max_batch * 8), "cudaMallocHost");
		check_cuda(cudaMallocHost((void **) &sl->offs_h, ((size_t) s->opts.max_batch + 1) * 8), "cudaMallocHost");
		ts->slots.push_back(std::move(sl));
	}
	std::lock_guard<std::mutex> lk(s->mu);
	s->trees.push_back(std::move(ts));
	return (uint32_t) s->trees.size() - 1;
}

void server_submit(Server *s, uint32_t n, const uint32_t *tree_index, const pst_query *q, pst_ret ret,
                   const uint64_t *arrival_ns, uint64_t *ids)
{
	const uint64_t now = now_ns();
	{
		std::lock_guard<std::mutex> lk(s->mu);
		if (!s->worker_error.empty())
			fail(PST_ERR_INTERNAL, "server worker stopped: " + s->worker_error);
		for (uint32_t i = 0; i < n; i++) {
			const uint32_t t = tree_index ? tree_index[i] : 0;
			if (t >= s->trees.size())
				fail(PST_ERR_INVALID, "tree index out of range");
			if (q[i].kind < PST_Q_THREE || q[i].kind > PST_Q_RIGHT)
				fail(PST_ERR_INVALID, "query kind must be PST_Q_THREE, PST_Q_LEFT or PST_Q_RIGHT");
			if (ret == PST_RET_IDS && s->trees[t]->tree->idtype != PST_ID_U32)
				fail(PST_ERR_UNSUPPORTED, "an id-less tree can only return points");
		}
		for (uint32_t i = 0; i < n; i++) {
			auto r = std::make_unique<Request>();
			r->id = s->next_id++;
			r->tree = tree_index ? tree_index[i] : 0;
			r->q = q[i];
			r->ret = ret;
			r->arrival_ns = arrival_ns && arrival_ns[i] ? arrival_ns[i] : now;
			if (ids)
				ids[i] = r->id;
			s->inbox.push_back(r.get());
			s->reqs.emplace(r->id, std::move(r));
			s->outstanding++;
			s->st.submitted++;
		}
	}
	s->cv_work.notify_one();
}

pst_status server_wait(Server *s, uint64_t id, uint32_t timeout_ms, pst_status *status, uint64_t *count)
{
	std::unique_lock<std::mutex> lk(s->mu);
	auto it = s->reqs.find(id);
	if (it == s->reqs.end())
		fail(PST_ERR_INVALID, "unknown request id");
	Request *r = it->second.get();
	if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return r->state == REQ_DONE; }))
		return PST_ERR_TIMEOUT;
	if (status)
		*status = r->cancelled ? PST_ERR_INVALID : r->status;
	if (count)
		*count = r->count;
	return PST_OK;
}

pst_status server_take(Server *s, uint64_t id, void *host_out, uint64_t capacity, uint64_t *count)
{
	std::lock_guard<std::mutex> lk(s->mu);
	auto it = s->reqs.find(id);
	if (it == s->reqs.end())
		fail(PST_ERR_INVALID, "unknown request id");
	Request *r = it->second.get();
	if (r->state != REQ_DONE)
		return PST_ERR_BUSY;
	if (count)
		*count = r->count;
	if (host_out) {
		if (s->opts.keep_results != 1)
			fail(PST_ERR_UNSUPPORTED, "server created without keep_results = 1");
		if (r->count > capacity)
			return PST_ERR_CAPACITY;
		memcpy(host_out, r->result.data(), r->result.size());
	}
	const pst_status st = r->status;
	s->reqs.erase(it);
	return st;
}

pst_status server_cancel(Server *s, uint64_t id)
{
	std::lock_guard<std::mutex> lk(s->mu);
	auto it = s->reqs.find(id);
	if (it == s->reqs.end())
		fail(PST_ERR_INVALID, "unknown request id");
	if (it->second->state != REQ_DONE)
		it->second->cancelled = true;
	return PST_OK;
}

pst_status server_drain(Server *s, uint32_t timeout_ms)
{
	std::unique_lock<std::mutex> lk(s->mu);
	if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms),
	                         [&] { return s->outstanding == 0 || !s->worker_error.empty(); }))
		return PST_ERR_TIMEOUT;
	if (!s->worker_error.empty())
		fail(PST_ERR_INTERNAL, "server worker stopped: " + s->worker_error);
	return PST_OK;
}

void server_stats(Server *s, pst_server_stats *out)
{
	std::lock_guard<std::mutex> lk(s->mu);
	pst_server_stats st = s->st;
	std::vector<double> v = s->lat_ms;
	std::sort(v.begin(), v.end());
	auto pct = [&](double p) {
		if (v.empty())
			return 0.0;
		size_t i = (size_t) std::min<double>(v.size() - 1, std::max(0.0, p * (double) v.size() - 1e-9));
		return v[i];
	};
	st.p50_ms = pct(0.50);
	st.p90_ms = pct(0.90);
	st.p99_ms = pct(0.99);
	st.max_ms = v.empty() ? 0.0 : v.back();
	double sum = 0;
	for (double x : v)
		sum += x;
	st.mean_ms = v.empty() ? 0.0 : sum / (double) v.size();
	st.busy_s = s->last_done > s->first_arrival ? (double) (s->last_done - s->first_arrival) / 1e9 : 0.0;
	st.worker_cpu_s = (double) (s->worker_cpu_ns.load() - s->worker_cpu_base) / 1e9;
	*out = st;
}

void server_reset_stats(Server *s)
{
	std::lock_guard<std::mutex> lk(s->mu);
	const uint64_t keep_sub = s->st.submitted;
	s->st = pst_server_stats{};
	s->st.submitted = keep_sub;
	s->lat_ms.clear();
	s->first_arrival = s->last_done = 0;
	s->arena.peak = s->arena.used;
	s->worker_cpu_base = s->worker_cpu_ns.load();
}

void server_destroy(Server *s) { delete s; }

}  // namespace pst

// ---------------------------------------------------------------------------

struct pst_server {
	pst::Server *s;
};

namespace pst {
pst_status guarded_call(const std::function<void()> &f);
}

extern "C" {

pst_status pst_server_create(pst_server **out, const pst_server_opts *opts)
{
	return pst::guarded_call([&] {
		if (!out)
			pst::fail(PST_ERR_INVALID, "null output");
		pst_server_opts o{};
		if (opts)
			o = *opts;
		else
			o.use_graph = 1;
		auto *h = new pst_server{nullptr};
		try {
			h->s = pst::server_create(o);
		} catch (...) {
			delete h;
			throw;
		}
		*out = h;
	});
}

pst_status pst_server_add_tree(pst_server *srv, pst_tree *tree, uint32_t *tree_index)
{
	return pst_server_add_tree_tuned(srv, tree, nullptr, tree_index);
}

pst_status pst_server_add_tree_tuned(pst_server *srv, pst_tree *tree, const pst_batch_opts *tuning,
                                     uint32_t *tree_index)
{
	return pst::guarded_call([&] {
		if (!srv || !tree)
			pst::fail(PST_ERR_INVALID, "null argument");
		if (tree->t.n == 0)
			pst::fail(PST_ERR_INVALID, "an empty tree cannot be served");
		const uint32_t i = pst::server_add_tree(srv->s, &tree->t, tuning);
		if (tree_index)
			*tree_index = i;
	});
}

pst_status pst_server_submit(pst_server *srv, uint32_t n, const uint32_t *tree_index, const pst_query *queries,
                             pst_ret ret, const uint64_t *arrival_ns, uint64_t *ids)
{
	return pst::guarded_call([&] {
		if (!srv || (n && !queries))
			pst::fail(PST_ERR_INVALID, "null argument");
		if (ret != PST_RET_IDS && ret != PST_RET_POINTS)
			pst::fail(PST_ERR_INVALID, "bad return type");
		pst::server_submit(srv->s, n, tree_index, queries, ret, arrival_ns, ids);
	});
}

pst_status pst_server_wait(pst_server *srv, uint64_t id, uint32_t timeout_ms, pst_status *status, uint64_t *count)
{
	pst_status r = PST_OK;
	pst_status st = pst::guarded_call([&] {
		if (!srv)
			pst::fail(PST_ERR_INVALID, "null server");
		r = pst::server_wait(srv->s, id, timeout_ms, status, count);
	});
	return st != PST_OK ? st : r;
}

pst_status pst_server_take(pst_server *srv, uint64_t id, void *host_out, uint64_t capacity, uint64_t *count)
{
	pst_status r = PST_OK;
	pst_status st = pst::guarded_call([&] {
		if (!srv)
			pst::fail(PST_ERR_INVALID, "null server");
		r = pst::server_take(srv->s, id, host_out, capacity, count);
	});
	return st != PST_OK ? st : r;
}

pst_status pst_server_cancel(pst_server *srv, uint64_t id)
{
	return pst::guarded_call([&] {
		if (!srv)
			pst::fail(PST_ERR_INVALID, "null server");
		pst::server_cancel(srv->s, id);
	});
}

pst_status pst_server_drain(pst_server *srv, uint32_t timeout_ms)
{
	pst_status r = PST_OK;
	pst_status st = pst::guarded_call([&] {
		if (!srv)
			pst::fail(PST_ERR_INVALID, "null server");
		r = pst::server_drain(srv->s, timeout_ms);
	});
	return st != PST_OK ? st : r;
}

pst_status pst_server_get_stats(pst_server *srv, pst_server_stats *stats)
{
	return pst::guarded_call([&] {
		if (!srv || !stats)
			pst::fail(PST_ERR_INVALID, "null argument");
		pst::server_stats(srv->s, stats);
	});
}

pst_status pst_server_reset_stats(pst_server *srv)
{
	return pst::guarded_call([&] {
		if (!srv)
			pst::fail(PST_ERR_INVALID, "null server");
		pst::server_reset_stats(srv->s);
	});
}

pst_status pst_server_destroy(pst_server *srv)
{
	return pst::guarded_call([&] {
		if (!srv)
			return;
		pst::server_destroy(srv->s);
		delete srv;
	});
}

}  // extern "C"
