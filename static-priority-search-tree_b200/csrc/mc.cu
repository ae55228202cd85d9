// Marching cubes over active metacells: the isosurface stage after the PST query.
// The query gives the metacells whose [min, max] contains the isovalue; every cell
// (voxel cube) of those metacells is classified by its 8 corner values and turned
// into triangles.  Headless: triangles go to a device buffer (9 float32 each, three
// vertices in vertex-index units).
//
// The triangle table is derived here from first principles (no third-party table):
//   * corner c of a cell sits at (c & 1, c >> 1 & 1, c >> 2 & 1); edge 4a + u + 2v runs
//     along axis a at the other two coordinates (u, v); a corner is inside when its
//     value is >= iso;
//   * on each cell face the edges whose ends differ are joined in pairs: two such
//     edges by one segment; four (diagonal corners inside) by two segments that each
//     cut off one inside corner.  A face decides alone, so the two cells sharing it
//     agree and the surface is closed;
//   * every crossed edge then has two segment ends, so the segments form loops; a
//     loop is oriented so that its (Newell) normal points from the inside ends of its
//     edges to the outside ends, rotated to start at its smallest edge, and fanned
//     from the first vertex whose diagonals all leave the cube faces (a diagonal on a
//     face would overlap the neighbouring cell).  At most 5 triangles per cell.
// Vertices: on the edge from global vertex a (the lower end) to b,
// t = (iso - f_a) / (f_b - f_a) and the coordinate along the edge's axis is a + t,
// rounded IEEE operations with nothing fused, so a vertex shared by neighbouring
// cells has the same bits in both.
//
// Kernels (k_mc_cells): one warp per metacell, 32 cells at a time; the count pass
// sums each metacell's triangles, an exclusive scan gives offsets, the emit pass
// computes each cell's triangles at its warp-scanned position in a per-warp shared
// stage and writes the 32 cells' triangles out as one contiguous run, so the output is
// ordered by metacell (as given), then cell (x fastest), then table order.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "scan_sort.cuh"
#include "tree.cuh"

namespace pst {

namespace {

constexpr int MC_MAX_TRI = 5;

struct McTables {
	uint8_t ntri[256];
	uint8_t edges[256][3 * MC_MAX_TRI];
};

// ---------------------------------------------------------------------------
// Table generation (host).

struct Geometry {
	int corner[8][3];
	int edge[12][2];
	int axis[12];
	int face[6][4];  // corners in ring order

	Geometry()
	{
		for (int c = 0; c < 8; c++) {
			corner[c][0] = c & 1;
			corner[c][1] = (c >> 1) & 1;
			corner[c][2] = (c >> 2) & 1;
		}
		int e = 0;
		for (int a = 0; a < 3; a++) {
			const int o0 = a == 0 ? 1 : 0, o1 = a == 2 ? 1 : 2;
			for (int v = 0; v < 2; v++)
				for (int u = 0; u < 2; u++) {
					int lo[3] = {0, 0, 0};
					lo[o0] = u;
					lo[o1] = v;
					int hi[3] = {lo[0], lo[1], lo[2]};
					hi[a] = 1;
					edge[e][0] = lo[0] | (lo[1] << 1) | (lo[2] << 2);
					edge[e][1] = hi[0] | (hi[1] << 1) | (hi[2] << 2);
					axis[e] = a;
					e++;
				}
		}
		int f = 0;
		const int ring[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};
		for (int a = 0; a < 3; a++) {
			const int o0 = a == 0 ? 1 : 0, o1 = a == 2 ? 1 : 2;
			for (int s = 0; s < 2; s++) {
				for (int r = 0; r < 4; r++) {
					int p[3];
					p[a] = s;
					p[o0] = ring[r][0];
					p[o1] = ring[r][1];
					face[f][r] = p[0] | (p[1] << 1) | (p[2] << 2);
				}
				f++;
			}
		}
	}
	int edge_between(int c0, int c1) const
	{
		for (int e = 0; e < 12; e++)
			if ((edge[e][0] == c0 && edge[e][1] == c1) || (edge[e][0] == c1 && edge[e][1] == c0))
				return e;
		return -1;
	}
	unsigned faces_of_edge(int e) const
	{
		unsigned m = 0;
		for (int f = 0; f < 6; f++) {
			bool a = false, b = false;
			for (int r = 0; r < 4; r++) {
				a |= face[f][r] == edge[e][0];
				b |= face[f][r] == edge[e][1];
			}
			if (a && b)
				m |= 1u << f;
		}
		return m;
	}
};

void build_tables(McTables &T)
{
	const Geometry G;
	memset(&T, 0, sizeof(T));
	memset(T.edges, 255, sizeof(T.edges));
	for (int cfg = 0; cfg < 256; cfg++) {
		int inside[8];
		for (int c = 0; c < 8; c++)
			inside[c] = (cfg >> c) & 1;
		std::vector<int> adj[12];
		for (int f = 0; f < 6; f++) {
			int cut[4], xs[4], nx = 0;
			for (int i = 0; i < 4; i++) {
				cut[i] = G.edge_between(G.face[f][i], G.face[f][(i + 1) % 4]);
				if (inside[G.face[f][i]] != inside[G.face[f][(i + 1) % 4]])
					xs[nx++] = i;
			}
			auto join = [&](int a, int b) {
				adj[a].push_back(b);
				adj[b].push_back(a);
			};
			if (nx == 2)
				join(cut[xs[0]], cut[xs[1]]);
			else if (nx == 4)
				for (int i = 0; i < 4; i++)
					if (inside[G.face[f][i]])
						join(cut[(i + 3) % 4], cut[i]);
		}
		bool seen[12] = {};
		int ntri = 0;
		for (int e0 = 0; e0 < 12; e0++) {
			if (adj[e0].empty() || seen[e0])
				continue;
			std::vector<int> loop{e0};
			seen[e0] = true;
			int prev = -1, cur = e0, nxt = std::min(adj[e0][0], adj[e0][1]);
			while (nxt != e0) {
				loop.push_back(nxt);
				seen[nxt] = true;
				prev = cur;
				cur = nxt;
				nxt = adj[cur][0] != prev ? adj[cur][0] : adj[cur][1];
			}
			// orientation: Newell normal of the loop (twice the edge midpoints, integer)
			// against the inside-to-outside directions of its edges
			const int k = (int) loop.size();
			long nrm[3] = {0, 0, 0}, g[3] = {0, 0, 0};
			for (int i = 0; i < k; i++) {
				const int e = loop[i], e2 = loop[(i + 1) % k];
				long p[3], q[3];
				for (int d = 0; d < 3; d++) {
					p[d] = G.corner[G.edge[e][0]][d] + G.corner[G.edge[e][1]][d];
					q[d] = G.corner[G.edge[e2][0]][d] + G.corner[G.edge[e2][1]][d];
				}
				nrm[0] += p[1] * q[2] - p[2] * q[1];
				nrm[1] += p[2] * q[0] - p[0] * q[2];
				nrm[2] += p[0] * q[1] - p[1] * q[0];
				const int a = G.edge[e][0], b = G.edge[e][1];
				const int in = inside[a] ? a : b, out = inside[a] ? b : a;
				for (int d = 0; d < 3; d++)
					g[d] += G.corner[out][d] - G.corner[in][d];
			}
			const long dot = nrm[0] * g[0] + nrm[1] * g[1] + nrm[2] * g[2];
			if (dot == 0)
				fail(PST_ERR_INTERNAL, "marching-cubes table: degenerate loop");
			if (dot < 0)
				std::reverse(loop.begin(), loop.end());
			std::rotate(loop.begin(), std::min_element(loop.begin(), loop.end()), loop.end());
			// fan from the first vertex whose diagonals all leave the cube faces
			int apex = -1;
			for (int j = 0; j < k && apex < 0; j++) {
				bool ok = true;
				for (int i = 2; i < k - 1 && ok; i++)
					ok = (G.faces_of_edge(loop[j]) & G.faces_of_edge(loop[(j + i) % k])) == 0;
				if (ok)
					apex = j;
			}
			if (apex < 0)
				fail(PST_ERR_INTERNAL, "marching-cubes table: no valid fan");
			for (int i = 1; i < k - 1; i++) {
				if (ntri >= MC_MAX_TRI)
					fail(PST_ERR_INTERNAL, "marching-cubes table: too many triangles");
				T.edges[cfg][3 * ntri + 0] = (uint8_t) loop[apex];
				T.edges[cfg][3 * ntri + 1] = (uint8_t) loop[(apex + i) % k];
				T.edges[cfg][3 * ntri + 2] = (uint8_t) loop[(apex + i + 1) % k];
				ntri++;
			}
		}
		T.ntri[cfg] = (uint8_t) ntri;
	}
}

const McTables &host_tables()
{
	static McTables T;
	static std::once_flag once;
	std::call_once(once, [] { build_tables(T); });
	return T;
}

// ---------------------------------------------------------------------------
// Device side.

__constant__ McTables c_mc;
// corner offsets and edge ends, in the numbering above
__constant__ uint8_t c_edge_lo[12] = {0, 2, 4, 6, 0, 1, 4, 5, 0, 1, 2, 3};
__constant__ uint8_t c_edge_axis[12] = {0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 2};

std::mutex g_mc_mu;
bool g_mc_uploaded[64] = {};

void upload_tables()
{
	int dev = 0;
	PST_CUDA(cudaGetDevice(&dev));
	if (dev < 0 || dev >= 64)
		fail(PST_ERR_CUDA, "device index out of range");
	std::lock_guard<std::mutex> lk(g_mc_mu);
	if (g_mc_uploaded[dev])
		return;
	PST_CUDA(cudaMemcpyToSymbol(c_mc, &host_tables(), sizeof(McTables)));
	g_mc_uploaded[dev] = true;
}

struct McGrid {
	uint32_t px, py, pz, mcx, mcy, mcz, Mx, My;
};

constexpr int MC_THREADS = 128;
// Triangles a warp stages per 32 cells (at most MC_MAX_TRI each), 9 floats each.
constexpr int MC_STAGE_FLOATS = 32 * MC_MAX_TRI * 9;

template <bool EMIT>
__global__ void __launch_bounds__(MC_THREADS) k_mc_cells(const float *__restrict__ vol, McGrid g,
                                                  const uint32_t *__restrict__ ids, uint64_t n, float iso,
                                                  uint64_t *__restrict__ counts, const uint64_t *__restrict__ offsets,
                                                  float *__restrict__ tri, uint64_t capacity)
{
	__shared__ McTables s_t;
	// the warp's triangles of 32 cells, in output order, written out together
	__shared__ float s_tri[EMIT ? MC_THREADS / 32 : 1][EMIT ? MC_STAGE_FLOATS : 1];
	for (int i = threadIdx.x; i < (int) sizeof(McTables) / 4; i += blockDim.x)
		reinterpret_cast<uint32_t *>(&s_t)[i] = reinterpret_cast<const uint32_t *>(&c_mc)[i];
	__syncthreads();
	const uint32_t lane = threadIdx.x & 31;
	const uint64_t gw = ((uint64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nw = ((uint64_t) gridDim.x * blockDim.x) >> 5;
	const uint64_t plane = (uint64_t) g.px * g.py;
	for (uint64_t i = gw; i < n; i += nw) {
		const uint32_t id = ids[i];
		const uint32_t mx = id % g.Mx, my = (id / g.Mx) % g.My, mz = id / (g.Mx * g.My);
		const uint32_t x0 = mx * g.mcx, y0 = my * g.mcy, z0 = mz * g.mcz;
		const uint32_t nx = min(x0 + g.mcx, g.px - 1) - min(x0, g.px - 1);
		const uint32_t ny = min(y0 + g.mcy, g.py - 1) - min(y0, g.py - 1);
		const uint32_t nz = min(z0 + g.mcz, g.pz - 1) - min(z0, g.pz - 1);
		const uint32_t ncell = nx * ny * nz;
		uint64_t base = EMIT ? offsets[i] : 0;
		uint32_t total = 0;
		for (uint32_t c0 = 0; c0 < ncell; c0 += 32) {
			const uint32_t c = c0 + lane;
			float f[8];
			uint32_t cfg = 0, x = 0, y = 0, z = 0;
			if (c < ncell) {
				x = x0 + c % nx;
				y = y0 + (c / nx) % ny;
				z = z0 + c / (nx * ny);
				const float *p = vol + (uint64_t) z * plane + (uint64_t) y * g.px + x;
#pragma unroll
				for (int k = 0; k < 8; k++) {
					f[k] = p[(uint64_t) ((k >> 2) & 1) * plane + (uint64_t) ((k >> 1) & 1) * g.px + (k & 1)];
					cfg |= f[k] >= iso ? 1u << k : 0u;
				}
			}
			const uint32_t nt = c < ncell ? s_t.ntri[cfg] : 0u;
			if constexpr (!EMIT) {
				total += nt;
			} else {
				const uint32_t inc = warp_incl_scan(nt);
				const uint32_t tot = __shfl_sync(0xFFFFFFFFu, inc, 31);
				float *stage = s_tri[threadIdx.x >> 5];
				for (uint32_t k = 0; k < nt; k++) {
					float *dst = stage + (inc - nt + k) * 9;
#pragma unroll
					for (int v = 0; v < 3; v++) {
						const uint32_t e = s_t.edges[cfg][3 * k + v];
						const uint32_t a = c_edge_lo[e], ax = c_edge_axis[e];
						const uint32_t b = a | (1u << ax);
						const float t = __fdiv_rn(__fsub_rn(iso, f[a]), __fsub_rn(f[b], f[a]));
						float pos[3] = {(float) (x + (a & 1)), (float) (y + ((a >> 1) & 1)),
						                (float) (z + ((a >> 2) & 1))};
						pos[ax] = __fadd_rn(pos[ax], t);
						dst[3 * v + 0] = pos[0];
						dst[3 * v + 1] = pos[1];
						dst[3 * v + 2] = pos[2];
					}
				}
				__syncwarp();
				// the 32 cells' triangles are one contiguous range: consecutive lanes
				// write consecutive floats
				const uint64_t nf = (uint64_t) tot * 9;
				const uint64_t room = base < capacity ? (capacity - base) * 9 : 0;
				float *out = tri + base * 9;
				for (uint32_t j = lane; j < nf && j < room; j += 32)
					out[j] = stage[j];
				__syncwarp();  // the stage is refilled by the next 32 cells
				base += tot;
			}
		}
		if constexpr (!EMIT) {
#pragma unroll
			for (int o = 16; o > 0; o >>= 1)
				total += __shfl_xor_sync(0xFFFFFFFFu, total, o);
			if (lane == 0)
				counts[i] = total;
		}
	}
}

McGrid make_grid(const uint32_t P[3], const uint32_t mc[3])
{
	McGrid g;
	g.px = P[0];
	g.py = P[1];
	g.pz = P[2];
	g.mcx = mc[0];
	g.mcy = mc[1];
	g.mcz = mc[2];
	g.Mx = (P[0] - 1 + mc[0] - 1) / mc[0];
	g.My = (P[1] - 1 + mc[1] - 1) / mc[1];
	return g;
}

unsigned mc_grid_blocks(uint64_t n)
{
	const uint64_t want = (n + MC_THREADS / 32 - 1) / (MC_THREADS / 32);  // one metacell per warp
	return (unsigned) std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t) device_info().sms * 16));
}

}  // namespace

void mc_tables(uint8_t *ntri, uint8_t *edges)
{
	const McTables &T = host_tables();
	memcpy(ntri, T.ntri, 256);
	memcpy(edges, T.edges, sizeof(T.edges));
}

uint64_t mc_run(const float *vol, const uint32_t P[3], const uint32_t mc[3], const uint32_t *ids, uint64_t n, float iso,
                float *tri, uint64_t capacity, bool emit, cudaStream_t s)
{
	upload_tables();
	if (n == 0)
		return 0;
	const McGrid g = make_grid(P, mc);
	uint64_t *counts = nullptr, *offsets = nullptr, *scan = nullptr, *total_d = nullptr;
	const size_t tmp = scan_tmp_elems(n) * 8;
	char *buf = nullptr;
	const size_t bytes = n * 8 + (n + 1) * 8 + tmp + 64;
	cudaError_t e = cudaMallocAsync((void **) &buf, bytes, s);
	if (e == cudaErrorMemoryAllocation) {
		cudaGetLastError();
		fail(PST_ERR_NOMEM, "marching-cubes scratch of " + std::to_string(bytes) + " B failed");
	}
	check_cuda(e, "cudaMallocAsync(marching cubes)");
	struct Free {
		char *p;
		cudaStream_t s;
		~Free() { cudaFreeAsync(p, s); }
	} fr{buf, s};
	offsets = reinterpret_cast<uint64_t *>(buf);
	scan = reinterpret_cast<uint64_t *>(buf + (n + 1) * 8);
	total_d = reinterpret_cast<uint64_t *>(buf + (n + 1) * 8 + tmp);
	counts = reinterpret_cast<uint64_t *>(buf + (n + 1) * 8 + tmp + 64);
	const unsigned blocks = mc_grid_blocks(n);
	k_mc_cells<false><<<blocks, MC_THREADS, 0, s>>>(vol, g, ids, n, iso, counts, nullptr, nullptr, 0);
	PST_CUDA(cudaGetLastError());
	exclusive_scan<uint64_t>(counts, offsets, n, scan, total_d, s);
	uint64_t total = 0;
	PST_CUDA(cudaMemcpyAsync(&total, total_d, 8, cudaMemcpyDeviceToHost, s));
	PST_CUDA(cudaStreamSynchronize(s));
	if (!emit || total == 0 || total > capacity)
		return total;
	if (!tri)
		fail(PST_ERR_INVALID, "null triangle buffer");
	k_mc_cells<true><<<blocks, MC_THREADS, 0, s>>>(vol, g, ids, n, iso, nullptr, offsets, tri, capacity);
	PST_CUDA(cudaGetLastError());
	PST_CUDA(cudaStreamSynchronize(s));
	return total;
}

}  // namespace pst
