// Streaming kernels: the interval parallel search comparator and metacell formation.
#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "scan_kernels.cuh"

namespace pst {

namespace {

// ---------------------------------------------------------------------------
// Interval parallel search (interval-parallel-search/interval-parallel-search.h:76-117):
// report every point with dim1 <= v <= dim2.  A warp owns 256 consecutive records;
// each load instruction reads 32 consecutive records, ranks come from ballots in
// input order, and one atomic per 2048-record tile reserves the output, so the
// results of a tile keep their input order.

constexpr int IPS_THREADS = 256;
constexpr int IPS_PER_LANE = 8;
constexpr uint64_t IPS_WARP_SPAN = 32 * IPS_PER_LANE;
constexpr uint64_t IPS_TILE = IPS_WARP_SPAN * (IPS_THREADS / 32);

// Records of 4-byte values (8 or 12 bytes) would take two or three 4-byte loads per
// lane; a whole, 16-byte aligned warp span is instead copied with 16-byte cp.async
// into shared memory (two buffers per warp: the next tile's span is in flight while
// the current one is tested and written) and the lanes pick their records there.
template <typename Pt>
constexpr bool ips_staged() { return sizeof(Pt) <= 12 && (IPS_WARP_SPAN * sizeof(Pt)) % (16 * 32) == 0; }

// 16-byte copies per lane of one staged warp span, and the dynamic shared memory of
// k_ips (two spans per warp).
template <typename Pt>
constexpr int ips_vec() { return ips_staged<Pt>() ? (int) (IPS_WARP_SPAN * sizeof(Pt) / 16 / 32) : 0; }
template <typename Pt>
constexpr size_t ips_smem() { return (size_t) 2 * (IPS_THREADS / 32) * ips_vec<Pt>() * 32 * 16; }

template <typename T, bool HAS_ID, bool POINTS>
__global__ void __launch_bounds__(IPS_THREADS) k_ips(const Point<T, HAS_ID> *__restrict__ pts, uint64_t n, T v,
                                                    void *out, uint64_t capacity, unsigned long long *counter,
                                                    bool aligned16)
{
	using Pt = Point<T, HAS_ID>;
	constexpr bool STAGED = ips_staged<Pt>();
	constexpr int VEC = ips_vec<Pt>();
	extern __shared__ __align__(16) uint4 s_span[];  // [2][IPS_THREADS / 32][VEC * 32] when STAGED
	__shared__ uint32_t s_warp[IPS_THREADS / 32 + 1];
	__shared__ unsigned long long s_base;
	const int warp = threadIdx.x >> 5;
	const uint32_t lane = lane_id();
	const uint64_t tiles = (n + IPS_TILE - 1) / IPS_TILE;
	const bool staging = STAGED && aligned16;
	// a tile's span of this warp can be staged when it is whole
	auto whole = [&](uint64_t tl) { return tl < tiles && tl * IPS_TILE + (warp + 1) * IPS_WARP_SPAN <= n; };
	auto issue = [&](uint64_t tl, int b) {
		const uint4 *src = reinterpret_cast<const uint4 *>(pts + tl * IPS_TILE + warp * IPS_WARP_SPAN);
		uint4 *dst = s_span + ((size_t) b * (IPS_THREADS / 32) + warp) * (VEC * 32);
#pragma unroll
		for (int j = 0; j < VEC; j++)
			cp_async16(dst + j * 32 + lane, src + j * 32 + lane);
	};
	int cur = 0;
	bool staged_cur = false;
	if (staging) {
		staged_cur = whole(blockIdx.x);
		if (staged_cur)
			issue(blockIdx.x, 0);
		cp_async_commit();
	}
	for (uint64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
		const uint64_t wbase = tile * IPS_TILE + warp * IPS_WARP_SPAN;
		uint32_t hit[IPS_PER_LANE];
		Pt rec[IPS_PER_LANE];
		uint32_t wcount = 0;
		bool staged_next = false;
		if (staging) {
			staged_next = whole(tile + gridDim.x);
			if (staged_next)
				issue(tile + gridDim.x, cur ^ 1);
			cp_async_commit();
			cp_async_wait_group<1>();  // this tile's span has landed
			__syncwarp();
		}
		if (staged_cur) {
			const Pt *sp = reinterpret_cast<const Pt *>(s_span + ((size_t) cur * (IPS_THREADS / 32) + warp) * (VEC * 32));
#pragma unroll
			for (int k = 0; k < IPS_PER_LANE; k++) {
				rec[k] = sp[32 * k + lane];
				const bool ok = rec[k].dim1 <= v && v <= rec[k].dim2;
				hit[k] = __ballot_sync(0xFFFFFFFFu, ok);
				wcount += __popc(hit[k]);
			}
			__syncwarp();  // the buffer is refilled for the tile after next
		} else {
#pragma unroll
			for (int k = 0; k < IPS_PER_LANE; k++) {
				const uint64_t i = wbase + 32 * k + lane;
				bool ok = false;
				if (i < n) {
					rec[k] = pts[i];
					ok = rec[k].dim1 <= v && v <= rec[k].dim2;
				}
				hit[k] = __ballot_sync(0xFFFFFFFFu, ok);
				wcount += __popc(hit[k]);
			}
		}
		if (lane == 0)
			s_warp[warp] = wcount;
		__syncthreads();
		if (threadIdx.x == 0) {
			uint32_t run = 0;
			for (int w = 0; w < IPS_THREADS / 32; w++) {
				const uint32_t c = s_warp[w];
				s_warp[w] = run;
				run += c;
			}
			s_base = run ? atomicAdd(counter, (unsigned long long) run) : 0ull;
		}
		__syncthreads();
		uint64_t o = s_base + s_warp[warp];
#pragma unroll
		for (int k = 0; k < IPS_PER_LANE; k++) {
			if ((hit[k] >> lane) & 1u) {
				const uint64_t pos = o + __popc(hit[k] & lanemask_lt());
				if (pos < capacity) {
					if constexpr (POINTS)
						static_cast<Pt *>(out)[pos] = rec[k];
					else
						static_cast<uint32_t *>(out)[pos] = rec[k].id;
				}
			}
			o += __popc(hit[k]);
		}
		__syncthreads();
		staged_cur = staged_next;
		cur ^= 1;
	}
	if (staging)
		cp_async_wait_all();  // nothing may still target this CTA's shared memory
}

// ---------------------------------------------------------------------------
// Metacell formation (helpers/isosurface-data-processing.tu:9-127, :181-212).
// Thread x of a CTA owns metacell column (mx = x, my) and walks a slab of metacells
// in z.  Vertex rows are read with consecutive threads on consecutive metacells;
// the shared boundary plane between consecutive metacells in z is reduced once and
// reused.

template <typename T>
__device__ __forceinline__ void plane_minmax(const T *__restrict__ vol, uint64_t px, uint64_t py, uint64_t z,
                                             uint32_t x0, uint32_t x1, uint32_t y0, uint32_t y1, T &lo, T &hi)
{
	const T *plane = vol + z * py * px;
	lo = hi = plane[(uint64_t) y0 * px + x0];
	for (uint32_t y = y0; y <= y1; y++) {
		const T *row = plane + (uint64_t) y * px;
		for (uint32_t x = x0; x <= x1; x++) {
			const T val = row[x];
			lo = val < lo ? val : lo;
			hi = val > hi ? val : hi;
		}
	}
}

// Metacell layers [mz_begin, mz_end); `vol` holds the vertex planes from z_base on
// (the whole volume: z_base = 0; one z-slab of it: its first plane).
template <typename T, bool HAS_ID>
__global__ void k_metacells(const T *__restrict__ vol, uint32_t px, uint32_t py, uint32_t pz, uint32_t mcx,
                            uint32_t mcy, uint32_t mcz, uint32_t Mx, uint32_t My, uint32_t mz_begin, uint32_t mz_end,
                            uint32_t z_base, uint32_t mz_per_cta, Point<T, HAS_ID> *__restrict__ out)
{
	const uint32_t mx = blockIdx.x * blockDim.x + threadIdx.x;
	const uint32_t my = blockIdx.y;
	const uint32_t mz0 = mz_begin + blockIdx.z * mz_per_cta;
	const uint32_t mz1 = min(mz0 + mz_per_cta, mz_end);
	if (mx >= Mx)
		return;
	const uint32_t x0 = mx * mcx, x1 = min(x0 + mcx, px - 1);
	const uint32_t y0 = my * mcy, y1 = min(y0 + mcy, py - 1);
	T plo = T(0), phi = T(0);     // the last plane reduced
	uint32_t pz_done = 0xFFFFFFFFu;
	for (uint32_t mz = mz0; mz < mz1; mz++) {
		const uint32_t z0 = mz * mcz, z1 = min(z0 + mcz, pz - 1);
		T lo, hi;
		if (pz_done == z0) {
			lo = plo;
			hi = phi;
		} else {
			plane_minmax(vol, px, py, z0 - z_base, x0, x1, y0, y1, lo, hi);
		}
		for (uint32_t z = z0 + 1; z <= z1; z++) {
			plane_minmax(vol, px, py, z - z_base, x0, x1, y0, y1, plo, phi);
			lo = plo < lo ? plo : lo;
			hi = phi > hi ? phi : hi;
			pz_done = z;
		}
		const uint64_t id = (uint64_t) mx + ((uint64_t) my + (uint64_t) mz * My) * Mx;
		Point<T, HAS_ID> p;
		p.dim1 = lo;
		p.dim2 = hi;
		if constexpr (HAS_ID)
			p.id = (uint32_t) id;
		out[id] = p;
	}
}

// The common layout: metacells 4 vertices wide over 4-byte values, rows a multiple of
// 4 vertices long, the volume 16-byte aligned.  A metacell's 4 low vertices of a row
// are one aligned 16-byte load; its fifth (the next metacell's first) comes from the
// next lane, or from memory for a warp's last metacell.  Same walk as k_metacells.
template <typename T>
struct Quad;
template <>
struct Quad<float> {
	using V = float4;
};
template <>
struct Quad<int32_t> {
	using V = int4;
};

template <typename T, bool HAS_ID>
__global__ void k_metacells4(const T *__restrict__ vol, uint32_t px, uint32_t py, uint32_t pz, uint32_t mcy,
                             uint32_t mcz, uint32_t Mx, uint32_t My, uint32_t mz_begin, uint32_t mz_end,
                             uint32_t z_base, uint32_t mz_per_cta, Point<T, HAS_ID> *__restrict__ out)
{
	using V = typename Quad<T>::V;
	const uint32_t mx = blockIdx.x * blockDim.x + threadIdx.x;
	const uint32_t lane = lane_id();
	const bool active = mx < Mx;  // inactive lanes still take part in the shuffles
	const uint32_t my = blockIdx.y;
	const uint32_t mz0 = mz_begin + blockIdx.z * mz_per_cta;
	const uint32_t mz1 = min(mz0 + mz_per_cta, mz_end);
	const uint32_t x0 = 4 * mx;
	const bool has5 = active && x0 + 4 <= px - 1;         // the metacell has a fifth vertex column
	const bool from_next = lane < 31 && mx + 1 < Mx;     // ... and the next lane holds it
	const uint32_t y0 = my * mcy, y1 = min(y0 + mcy, py - 1);
	auto plane = [&](uint32_t z, T &lo, T &hi) {
		const T *pl = vol + (uint64_t) (z - z_base) * py * px;
		for (uint32_t y = y0; y <= y1; y++) {
			const T *row = pl + (uint64_t) y * px;
			const V a = active ? *reinterpret_cast<const V *>(row + x0) : V{};
			const T nx = __shfl_down_sync(0xFFFFFFFFu, a.x, 1);
			const T e = from_next ? nx : has5 ? row[x0 + 4] : a.x;
			// folds in row-major order that keep the first of equal values (as
			// k_metacells does), so -0.0 and +0.0 come out as they do there
			const T r[5] = {a.x, a.y, a.z, a.w, e};
			T l = r[0], h = r[0];
#pragma unroll
			for (int k = 1; k < 5; k++) {
				l = r[k] < l ? r[k] : l;
				h = r[k] > h ? r[k] : h;
			}
			if (y == y0) {
				lo = l;
				hi = h;
			} else {
				lo = l < lo ? l : lo;
				hi = h > hi ? h : hi;
			}
		}
	};
	T plo = T(0), phi = T(0);  // the last plane reduced
	uint32_t pz_done = 0xFFFFFFFFu;
	for (uint32_t mz = mz0; mz < mz1; mz++) {
		const uint32_t z0 = mz * mcz, z1 = min(z0 + mcz, pz - 1);
		T lo, hi;
		if (pz_done == z0) {
			lo = plo;
			hi = phi;
		} else {
			plane(z0, lo, hi);
		}
		for (uint32_t z = z0 + 1; z <= z1; z++) {
			plane(z, plo, phi);
			lo = plo < lo ? plo : lo;
			hi = phi > hi ? phi : hi;
			pz_done = z;
		}
		if (active) {
			const uint64_t id = (uint64_t) mx + ((uint64_t) my + (uint64_t) mz * My) * Mx;
			Point<T, HAS_ID> p;
			p.dim1 = lo;
			p.dim2 = hi;
			if constexpr (HAS_ID)
				p.id = (uint32_t) id;
			out[id] = p;
		}
	}
}

template <typename T, bool HAS_ID, bool POINTS>
void ips_launch(const void *pts, uint64_t n, T v, void *out, uint64_t cap, unsigned long long *counter,
                uint32_t blocks, cudaStream_t s)
{
	const uint64_t tiles = (n + IPS_TILE - 1) / IPS_TILE;
	uint64_t g = blocks ? blocks : std::min<uint64_t>(tiles, (uint64_t) device_info().sms * 8);
	g = std::max<uint64_t>(g, 1);
	const bool aligned16 = (reinterpret_cast<uintptr_t>(pts) & 15u) == 0;
	constexpr size_t smem = ips_smem<Point<T, HAS_ID>>();
	if (smem > 0) {
		// above the default 48 KB with the static part: opt in once per device
		static std::mutex mu;
		static bool done[64] = {};
		const int dev = device_info().device;
		std::lock_guard<std::mutex> lk(mu);
		if (dev >= 0 && dev < 64 && !done[dev]) {
			PST_CUDA(cudaFuncSetAttribute(k_ips<T, HAS_ID, POINTS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
			                              (int) smem));
			done[dev] = true;
		}
	}
	k_ips<T, HAS_ID, POINTS><<<(unsigned) g, IPS_THREADS, smem, s>>>(static_cast<const Point<T, HAS_ID> *>(pts), n, v,
	                                                                  out, cap, counter, aligned16);
	PST_CUDA(cudaGetLastError());
}

template <typename T>
void ips_dispatch(pst_idtype it, pst_ret ret, const void *pts, uint64_t n, T v, void *out, uint64_t cap,
                  unsigned long long *counter, uint32_t blocks, cudaStream_t s)
{
	if (ret == PST_RET_IDS) {
		if (it != PST_ID_U32)
			fail(PST_ERR_UNSUPPORTED, "id-less points can only be returned as points");
		ips_launch<T, true, false>(pts, n, v, out, cap, counter, blocks, s);
	} else if (it == PST_ID_U32) {
		ips_launch<T, true, true>(pts, n, v, out, cap, counter, blocks, s);
	} else {
		ips_launch<T, false, true>(pts, n, v, out, cap, counter, blocks, s);
	}
}

template <typename T, bool HAS_ID>
void metacell_launch(const void *vol, const uint32_t P[3], const uint32_t mc[3], const uint32_t M[3],
                     uint32_t mz_begin, uint32_t mz_end, void *out, cudaStream_t s)
{
	if (mz_end <= mz_begin)
		return;
	const uint32_t threads = M[0] >= 256 ? 256 : ((M[0] + 31) / 32) * 32;
	const uint32_t mzp = 8;
	dim3 grid((M[0] + threads - 1) / threads, M[1], (mz_end - mz_begin + mzp - 1) / mzp);
	if (grid.y > 65535 || grid.z > 65535)
		fail(PST_ERR_INVALID, "metacell grid too large");
	bool quad = false;
	if constexpr (sizeof(T) == 4)
		quad = mc[0] == 4 && P[0] % 4 == 0 && (reinterpret_cast<uintptr_t>(vol) & 15u) == 0;
	if constexpr (sizeof(T) == 4) {
		if (quad)
			k_metacells4<T, HAS_ID><<<grid, threads, 0, s>>>(static_cast<const T *>(vol), P[0], P[1], P[2], mc[1], mc[2],
			                                                 M[0], M[1], mz_begin, mz_end, mz_begin * mc[2], mzp,
			                                                 static_cast<Point<T, HAS_ID> *>(out));
	}
	if (!quad)
		k_metacells<T, HAS_ID><<<grid, threads, 0, s>>>(static_cast<const T *>(vol), P[0], P[1], P[2], mc[0], mc[1],
		                                                mc[2], M[0], M[1], mz_begin, mz_end, mz_begin * mc[2], mzp,
		                                                static_cast<Point<T, HAS_ID> *>(out));
	PST_CUDA(cudaGetLastError());
}

}  // namespace

void ips_run(pst_dtype dt, pst_idtype it, pst_ret ret, const void *pts, uint64_t n, pst_value v, void *out,
             uint64_t cap, unsigned long long *counter_d, uint32_t blocks, cudaStream_t s)
{
	switch (dt) {
	case PST_F32: ips_dispatch<float>(it, ret, pts, n, v.f32, out, cap, counter_d, blocks, s); break;
	case PST_F64: ips_dispatch<double>(it, ret, pts, n, v.f64, out, cap, counter_d, blocks, s); break;
	case PST_I32: ips_dispatch<int32_t>(it, ret, pts, n, v.i32, out, cap, counter_d, blocks, s); break;
	default: fail(PST_ERR_INVALID, "bad dtype");
	}
}

void metacells_run_layers(pst_dtype dt, pst_idtype it, const void *vol, const uint32_t P[3], const uint32_t mc[3],
                          const uint32_t M[3], uint32_t mz_begin, uint32_t mz_end, void *out, cudaStream_t s)
{
	const bool id = it == PST_ID_U32;
	const uint32_t b = mz_begin, e = mz_end;
	switch (dt) {
	case PST_F32: id ? metacell_launch<float, true>(vol, P, mc, M, b, e, out, s) : metacell_launch<float, false>(vol, P, mc, M, b, e, out, s); break;
	case PST_F64: id ? metacell_launch<double, true>(vol, P, mc, M, b, e, out, s) : metacell_launch<double, false>(vol, P, mc, M, b, e, out, s); break;
	case PST_I32: id ? metacell_launch<int32_t, true>(vol, P, mc, M, b, e, out, s) : metacell_launch<int32_t, false>(vol, P, mc, M, b, e, out, s); break;
	default: fail(PST_ERR_INVALID, "bad dtype");
	}
}

void metacells_run(pst_dtype dt, pst_idtype it, const void *vol, const uint32_t P[3], const uint32_t mc[3],
                   const uint32_t M[3], void *out, cudaStream_t s)
{
	metacells_run_layers(dt, it, vol, P, mc, M, 0, M[2], out, s);
}

}  // namespace pst
