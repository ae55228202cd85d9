// Tree images: save a built tree and load it back without rebuilding (for a
// serving loop that restarts with the same resident trees).  The image is a 64-byte
// header followed by the tree's single device allocation byte for byte, so a load
// is one allocation and one copy; files stream through pinned double buffers, the
// disk transfer of one chunk overlapping the host-device copy of the previous one.
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>

#include "tree.cuh"

namespace pst {

namespace {

constexpr char MAGIC[8] = {'P', 'S', 'T', 'B', '2', '0', '0', 'T'};
constexpr uint32_t IMAGE_VERSION = 1;
constexpr uint64_t HEADER_BYTES = 64;
constexpr uint64_t FILE_CHUNK = 64ull << 20;  // pinned staging chunk

struct Header {
	char magic[8];
	uint32_t version;
	int32_t dtype;
	int32_t idtype;
	uint32_t levels;
	uint64_t n;
	uint64_t image_bytes;
	uint64_t header_bytes;
	uint8_t reserved[16];
};
static_assert(sizeof(Header) == HEADER_BYTES, "image header");

Header make_header(const TreeStorage &t)
{
	Header h{};
	memcpy(h.magic, MAGIC, 8);
	h.version = IMAGE_VERSION;
	h.dtype = t.dtype;
	h.idtype = t.idtype;
	h.levels = t.levels;
	h.n = t.n;
	h.image_bytes = t.bytes;
	h.header_bytes = HEADER_BYTES;
	return h;
}

// Validates a header and sets up t (dtype, idtype, n, levels); returns the image size.
uint64_t accept_header(TreeStorage &t, const Header &h)
{
	if (memcmp(h.magic, MAGIC, 8) != 0)
		fail(PST_ERR_INVALID, "not a tree image (bad magic)");
	if (h.version != IMAGE_VERSION || h.header_bytes != HEADER_BYTES)
		fail(PST_ERR_UNSUPPORTED, "tree image version " + std::to_string(h.version) + " is not supported");
	if (point_size(static_cast<pst_dtype>(h.dtype), static_cast<pst_idtype>(h.idtype)) == 0)
		fail(PST_ERR_INVALID, "tree image with an unknown value or id type");
	if (h.n >= (1ull << 31))
		fail(PST_ERR_INVALID, "tree image with more than 2^31 - 1 points");
	t.dtype = static_cast<pst_dtype>(h.dtype);
	t.idtype = static_cast<pst_idtype>(h.idtype);
	t.n = h.n;
	t.levels = tree_levels(h.n);
	if (t.levels != h.levels || tree_bytes(t.dtype, t.idtype, t.n) != h.image_bytes)
		fail(PST_ERR_INVALID, "tree image sizes do not match its point count");
	return h.image_bytes;
}

void allocate(TreeStorage &t, uint64_t bytes)
{
	if (!bytes)
		return;
	void *mem = nullptr;
	cudaError_t e = cudaMalloc(&mem, bytes);
	if (e == cudaErrorMemoryAllocation) {
		cudaGetLastError();
		fail(PST_ERR_NOMEM, "tree allocation of " + std::to_string(bytes) + " B failed");
	}
	check_cuda(e, "cudaMalloc(tree)");
	attach_tree_memory(t, mem);
}

struct PinnedPair {
	unsigned char *buf[2] = {nullptr, nullptr};
	cudaEvent_t done[2] = {nullptr, nullptr};
	explicit PinnedPair(uint64_t bytes)
	{
		for (int i = 0; i < 2; i++) {
			check_cuda(cudaMallocHost((void **) &buf[i], bytes), "cudaMallocHost(image staging)");
			check_cuda(cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming), "cudaEventCreate");
		}
	}
	~PinnedPair()
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

struct File {
	FILE *f = nullptr;
	File(const char *path, const char *mode) : f(fopen(path, mode))
	{
		if (!f)
			fail(PST_ERR_INVALID, std::string("cannot open ") + path);
	}
	~File()
	{
		if (f)
			fclose(f);
	}
};

}  // namespace

uint64_t serialized_size(const TreeStorage &t) { return HEADER_BYTES + t.bytes; }

void save_tree(const TreeStorage &t, void *host, uint64_t capacity, cudaStream_t s)
{
	const uint64_t need = serialized_size(t);
	if (!host || capacity < need)
		fail(PST_ERR_CAPACITY, "a tree image needs " + std::to_string(need) + " B");
	const Header h = make_header(t);
	memcpy(host, &h, HEADER_BYTES);
	if (t.bytes) {
		PST_CUDA(cudaMemcpyAsync(static_cast<unsigned char *>(host) + HEADER_BYTES, t.mem, t.bytes,
		                         cudaMemcpyDeviceToHost, s));
		PST_CUDA(cudaStreamSynchronize(s));
	}
}

void load_tree(TreeStorage &t, const void *host, uint64_t size, cudaStream_t s)
{
	if (!host || size < HEADER_BYTES)
		fail(PST_ERR_INVALID, "tree image shorter than its header");
	Header h;
	memcpy(&h, host, HEADER_BYTES);
	const uint64_t bytes = accept_header(t, h);
	if (size < HEADER_BYTES + bytes)
		fail(PST_ERR_INVALID, "tree image truncated");
	allocate(t, bytes);
	if (bytes) {
		try {
			PST_CUDA(cudaMemcpyAsync(t.mem, static_cast<const unsigned char *>(host) + HEADER_BYTES, bytes,
			                         cudaMemcpyHostToDevice, s));
			finish_tree_aux(t, s);
			PST_CUDA(cudaStreamSynchronize(s));
		} catch (...) {
			cudaStreamSynchronize(s);
			free_tree(t);
			throw;
		}
	}
}

void save_tree_file(const TreeStorage &t, const char *path)
{
	if (!path)
		fail(PST_ERR_INVALID, "null path");
	File f(path, "wb");
	const Header h = make_header(t);
	if (fwrite(&h, 1, HEADER_BYTES, f.f) != HEADER_BYTES)
		fail(PST_ERR_INVALID, std::string("write failed: ") + path);
	if (t.bytes) {
		cudaStream_t s;
		check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
		std::unique_ptr<CUstream_st, void (*)(cudaStream_t)> sguard(s, [](cudaStream_t x) { cudaStreamDestroy(x); });
		const uint64_t chunk = std::min<uint64_t>(FILE_CHUNK, t.bytes);
		PinnedPair pp(chunk);
		// copy chunk i+1 to the host while chunk i is written to disk
		const uint64_t nchunks = (t.bytes + chunk - 1) / chunk;
		auto issue = [&](uint64_t i) {
			const uint64_t off = i * chunk, len = std::min(chunk, t.bytes - off);
			PST_CUDA(cudaMemcpyAsync(pp.buf[i & 1], static_cast<const unsigned char *>(t.mem) + off, len,
			                         cudaMemcpyDeviceToHost, s));
			PST_CUDA(cudaEventRecord(pp.done[i & 1], s));
		};
		issue(0);
		for (uint64_t i = 0; i < nchunks; i++) {
			PST_CUDA(cudaEventSynchronize(pp.done[i & 1]));
			if (i + 1 < nchunks)
				issue(i + 1);
			const uint64_t off = i * chunk, len = std::min(chunk, t.bytes - off);
			if (fwrite(pp.buf[i & 1], 1, len, f.f) != len)
				fail(PST_ERR_INVALID, std::string("write failed: ") + path);
		}
	}
	if (fflush(f.f) != 0)
		fail(PST_ERR_INVALID, std::string("write failed: ") + path);
}

void load_tree_file(TreeStorage &t, const char *path, cudaStream_t s)
{
	if (!path)
		fail(PST_ERR_INVALID, "null path");
	File f(path, "rb");
	Header h;
	if (fread(&h, 1, HEADER_BYTES, f.f) != HEADER_BYTES)
		fail(PST_ERR_INVALID, std::string("tree image shorter than its header: ") + path);
	const uint64_t bytes = accept_header(t, h);
	allocate(t, bytes);
	if (!bytes)
		return;
	try {
		const uint64_t chunk = std::min<uint64_t>(FILE_CHUNK, bytes);
		PinnedPair pp(chunk);
		const uint64_t nchunks = (bytes + chunk - 1) / chunk;
		// read chunk i from disk while chunk i-1 is copied to the device
		for (uint64_t i = 0; i < nchunks; i++) {
			PST_CUDA(cudaEventSynchronize(pp.done[i & 1]));  // the buffer's previous copy is done
			const uint64_t off = i * chunk, len = std::min(chunk, bytes - off);
			if (fread(pp.buf[i & 1], 1, len, f.f) != len)
				fail(PST_ERR_INVALID, std::string("tree image truncated: ") + path);
			PST_CUDA(cudaMemcpyAsync(static_cast<unsigned char *>(t.mem) + off, pp.buf[i & 1], len,
			                         cudaMemcpyHostToDevice, s));
			PST_CUDA(cudaEventRecord(pp.done[i & 1], s));
		}
		finish_tree_aux(t, s);
		PST_CUDA(cudaStreamSynchronize(s));
	} catch (...) {
		cudaStreamSynchronize(s);
		free_tree(t);
		throw;
	}
}

}  // namespace pst
