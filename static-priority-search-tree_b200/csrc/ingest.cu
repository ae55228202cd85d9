// Volume ingest: raw scalar volumes (x fastest, then y, then z; no header -- the
// reference's readInVertices, helpers/isosurface-data-processing.h:205-229, reads
// them into host memory) streamed from disk to the device through pinned double
// buffers, the disk read of one chunk overlapping the host-to-device copy of the
// previous one; and metacell formation fused into the stream: each z-slab of
// metacell layers is reduced on the device while the next slab is read.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>

#include "scan_kernels.cuh"
#include "tree.cuh"

namespace pst {

namespace {

constexpr uint64_t DEFAULT_CHUNK = 64ull << 20;

struct File {
	FILE *f = nullptr;
	explicit File(const char *path) : f(fopen(path, "rb"))
	{
		if (!f)
			fail(PST_ERR_INVALID, std::string("failed to open ") + path + " for reading");
	}
	~File()
	{
		if (f)
			fclose(f);
	}
	void seek(uint64_t off, const char *path)
	{
		if (fseeko(f, (off_t) off, SEEK_SET) != 0)
			fail(PST_ERR_INVALID, std::string("seek failed in ") + path);
	}
	void read(void *dst, uint64_t bytes, uint64_t expected_total, const char *path)
	{
		const size_t got = fread(dst, 1, bytes, f);
		if (got != bytes)
			fail(PST_ERR_INVALID, std::string("short read of ") + path + ": expected " +
			                          std::to_string(expected_total) + " bytes");
	}
};

// Two pinned staging buffers with an event each marking the end of their last copy.
struct Staging {
	unsigned char *buf[2] = {nullptr, nullptr};
	cudaEvent_t done[2] = {nullptr, nullptr};
	explicit Staging(uint64_t bytes)
	{
		for (int i = 0; i < 2; i++) {
			check_cuda(cudaMallocHost((void **) &buf[i], std::max<uint64_t>(bytes, 16)), "cudaMallocHost(staging)");
			check_cuda(cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming), "cudaEventCreate");
		}
	}
	~Staging()
	{
		for (int i = 0; i < 2; i++) {
			if (done[i]) {
				cudaEventSynchronize(done[i]);
				cudaEventDestroy(done[i]);
			}
			if (buf[i])
				cudaFreeHost(buf[i]);
		}
	}
};

uint64_t file_size(File &f, const char *path)
{
	if (fseeko(f.f, 0, SEEK_END) != 0)
		fail(PST_ERR_INVALID, std::string("seek failed in ") + path);
	const off_t sz = ftello(f.f);
	f.seek(0, path);
	return (uint64_t) sz;
}

}  // namespace

void read_volume(const char *path, pst_dtype dt, uint64_t num_vertices, void *vert_d, cudaStream_t s)
{
	if (!path || !vert_d)
		fail(PST_ERR_INVALID, "null argument");
	const uint64_t bytes = num_vertices * value_size(dt);
	File f(path);
	if (file_size(f, path) < bytes)
		fail(PST_ERR_INVALID, std::string("short read of ") + path + ": expected " + std::to_string(bytes) + " bytes");
	if (!bytes)
		return;
	const uint64_t chunk = std::min(DEFAULT_CHUNK, bytes);
	Staging st(chunk);
	const uint64_t nchunks = (bytes + chunk - 1) / chunk;
	for (uint64_t i = 0; i < nchunks; i++) {
		PST_CUDA(cudaEventSynchronize(st.done[i & 1]));  // the buffer's previous copy has finished
		const uint64_t off = i * chunk, len = std::min(chunk, bytes - off);
		f.read(st.buf[i & 1], len, bytes, path);
		PST_CUDA(cudaMemcpyAsync(static_cast<unsigned char *>(vert_d) + off, st.buf[i & 1], len,
		                         cudaMemcpyHostToDevice, s));
		PST_CUDA(cudaEventRecord(st.done[i & 1], s));
	}
	PST_CUDA(cudaStreamSynchronize(s));
}

void metacells_from_file(const char *path, pst_dtype dt, pst_idtype it, const uint32_t P[3], const uint32_t mc[3],
                         const uint32_t M[3], void *out_d, uint64_t slab_bytes, cudaStream_t s)
{
	if (!path || !out_d)
		fail(PST_ERR_INVALID, "null argument");
	const uint64_t vs = value_size(dt);
	const uint64_t plane = (uint64_t) P[0] * P[1] * vs;
	const uint64_t total = plane * P[2];
	File f(path);
	if (file_size(f, path) < total)
		fail(PST_ERR_INVALID, std::string("short read of ") + path + ": expected " + std::to_string(total) + " bytes");
	if (!M[0] || !M[1] || !M[2])
		return;
	// metacell layers per slab: the slab holds its layers' vertex planes plus the
	// plane shared with the next slab
	const uint64_t want = slab_bytes ? slab_bytes : DEFAULT_CHUNK;
	uint64_t K = std::max<uint64_t>(1, want / std::max<uint64_t>(plane * mc[2], 1));
	K = std::min<uint64_t>(K, M[2]);
	const uint64_t slab_planes = K * mc[2] + 1;
	const uint64_t slab_cap = slab_planes * plane;
	Staging st(slab_cap);
	void *dev[2] = {nullptr, nullptr};
	struct DevFree {
		void **d;
		~DevFree()
		{
			for (int i = 0; i < 2; i++)
				if (d[i])
					cudaFree(d[i]);
		}
	} df{dev};
	for (int i = 0; i < 2; i++) {
		cudaError_t e = cudaMalloc(&dev[i], slab_cap);
		if (e == cudaErrorMemoryAllocation) {
			cudaGetLastError();
			fail(PST_ERR_NOMEM, "slab allocation of " + std::to_string(slab_cap) + " B failed");
		}
		check_cuda(e, "cudaMalloc(slab)");
	}
	const uint64_t nslabs = (M[2] + K - 1) / K;
	try {
		for (uint64_t j = 0; j < nslabs; j++) {
			const uint32_t mzb = (uint32_t) (j * K), mze = (uint32_t) std::min<uint64_t>((j + 1) * K, M[2]);
			const uint64_t z_lo = (uint64_t) mzb * mc[2];
			const uint64_t z_hi = std::min<uint64_t>((uint64_t) mze * mc[2], P[2] - 1);
			const uint64_t len = (z_hi - z_lo + 1) * plane;
			const int b = (int) (j & 1);
			// the staging buffer and the device slab of two slabs ago are free again
			PST_CUDA(cudaEventSynchronize(st.done[b]));
			f.seek(z_lo * plane, path);
			f.read(st.buf[b], len, total, path);
			PST_CUDA(cudaMemcpyAsync(dev[b], st.buf[b], len, cudaMemcpyHostToDevice, s));
			metacells_run_layers(dt, it, dev[b], P, mc, M, mzb, mze, out_d, s);
			PST_CUDA(cudaEventRecord(st.done[b], s));
		}
		PST_CUDA(cudaStreamSynchronize(s));
	} catch (...) {
		cudaStreamSynchronize(s);
		throw;
	}
}

}  // namespace pst
