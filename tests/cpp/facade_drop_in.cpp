// Drop-in check of the C++ facade: the calls the reference's testers make
// (testers/pst-tester-functions.tu:496-586, :711-736), written against
// static-pst-gpu.h, with results compared with a host brute force.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <sstream>
#include <vector>

#include "static-pst-gpu.h"

using Pt = PointStruct<float, unsigned, 1>;

#define CK(x)                                                                 \
	do {                                                                      \
		if ((x) != cudaSuccess) {                                             \
			std::fprintf(stderr, "CUDA error at %s:%d\n", __FILE__, __LINE__); \
			return 1;                                                         \
		}                                                                     \
	} while (0)

template <typename R>
static std::vector<R> fetch(R *d, size_t n)
{
	std::vector<R> h(n);
	if (n)
		cudaMemcpy(h.data(), d, n * sizeof(R), cudaMemcpyDeviceToHost);
	cudaFree(d);
	return h;
}

int main()
{
	const size_t n = 200000;
	std::mt19937 gen(1);
	std::uniform_real_distribution<float> u1(0.f, 1000.f), u2(0.f, 50.f);
	std::vector<Pt> pts(n);
	for (size_t i = 0; i < n; i++) {
		pts[i].dim1_val = u1(gen);
		pts[i].dim2_val = pts[i].dim1_val + u2(gen);
		pts[i].id = (unsigned) i;
	}
	Pt *pts_d;
	CK(cudaMalloc(&pts_d, n * sizeof(Pt)));
	CK(cudaMemcpy(pts_d, pts.data(), n * sizeof(Pt), cudaMemcpyHostToDevice));

	int failures = 0;
	auto brute = [&](int kind, float a, float b, float c) {
		std::vector<unsigned> r;
		for (auto &p : pts) {
			bool ok = c <= p.dim2_val &&
			          (kind == 0 ? (a <= p.dim1_val && p.dim1_val <= b) : kind == 1 ? p.dim1_val <= b : p.dim1_val >= a);
			if (ok)
				r.push_back(p.id);
		}
		std::sort(r.begin(), r.end());
		return r;
	};
	auto check = [&](const char *what, std::vector<unsigned> got, std::vector<unsigned> want) {
		std::sort(got.begin(), got.end());
		if (got != want) {
			std::printf("MISMATCH %s: %zu vs %zu\n", what, got.size(), want.size());
			failures++;
		}
	};

	{
		StaticPSTGPU<float, PointStruct, unsigned, 1> tree(pts_d, n);
		size_t k = 0;
		unsigned *ids_d = nullptr;
		tree.threeSidedSearch<unsigned>(k, ids_d, 400.f, 420.f, 430.f);
		check("threeSided ids", fetch(ids_d, k), brute(0, 400.f, 420.f, 430.f));
		Pt *pts_res = nullptr;
		tree.twoSidedLeftSearch(k, pts_res, 500.f, 500.f);  // default RetType = PointStruct
		auto pr = fetch(pts_res, k);
		std::vector<unsigned> pid;
		for (auto &p : pr) {
			if (!(p == pts[p.id]))
				failures++;
			pid.push_back(p.id);
		}
		check("twoSidedLeft points", pid, brute(1, 0.f, 500.f, 500.f));
		tree.twoSidedRightSearch<unsigned>(k, ids_d, 900.f, 940.f);
		check("twoSidedRight ids", fetch(ids_d, k), brute(2, 900.f, 0.f, 940.f));
		if (StaticPSTGPU<float, PointStruct, unsigned, 1>::calcGlobalMemNeeded(n) < n * 17)
			failures++;
	}
	{
		StaticPSTGPUArr<float, PointStruct, unsigned, 1> arr(pts_d, n, 128);
		size_t k = 0;
		unsigned *ids_d = nullptr;
		arr.twoSidedLeftSearch<unsigned>(k, ids_d, 300.f, 310.f);
		check("Arr twoSidedLeft", fetch(ids_d, k), brute(1, 0.f, 300.f, 310.f));
		arr.threeSidedSearch<unsigned>(k, ids_d, 10.f, 600.f, 550.f);
		check("Arr threeSided", fetch(ids_d, k), brute(0, 10.f, 600.f, 550.f));
	}
	{
		unsigned *ids_d = nullptr;
		size_t k = 0;
		intervalParallelSearch<float, PointStruct, unsigned, 1, unsigned>(pts_d, n, ids_d, k, 250.f, 0, 1, 32, 0, 128);
		check("IPS", fetch(ids_d, k), brute(1, 0.f, 250.f, 250.f));
	}
	{
		// empty tree: the reference's message and null result
		StaticPSTGPU<float, PointStruct, unsigned, 1> empty(pts_d, 0);
		size_t k = 7;
		unsigned *ids_d = reinterpret_cast<unsigned *>(1);
		empty.twoSidedLeftSearch<unsigned>(k, ids_d, 1.f, 1.f);
		if (k != 0 || ids_d != nullptr)
			failures++;
	}
	{
		// small tree printing through operator<< of the base class
		std::vector<Pt> few = {{3.f, 9.f, 0}, {1.f, 4.f, 1}, {2.f, 7.f, 2}};
		Pt *few_d;
		CK(cudaMalloc(&few_d, few.size() * sizeof(Pt)));
		CK(cudaMemcpy(few_d, few.data(), few.size() * sizeof(Pt), cudaMemcpyHostToDevice));
		StaticPSTGPU<float, PointStruct, unsigned, 1> t3(few_d, few.size());
		std::ostringstream os;
		os << t3;
		if (os.str().find("(3, 9; 1; 0)") == std::string::npos) {
			std::printf("unexpected print output:\n%s\n", os.str().c_str());
			failures++;
		}
		cudaFree(few_d);
	}
	{
		unsigned pd[3] = {33, 17, 9}, md[3] = {4, 4, 4}, g[3];
		size_t nm = 0;
		calcNumMetacells(pd, md, g, nm);
		std::vector<float> vol(33 * 17 * 9);
		for (size_t i = 0; i < vol.size(); i++)
			vol[i] = (float) ((i * 2654435761u) % 1000);
		float *vol_d;
		CK(cudaMalloc(&vol_d, vol.size() * sizeof(float)));
		CK(cudaMemcpy(vol_d, vol.data(), vol.size() * sizeof(float), cudaMemcpyHostToDevice));
		Pt *mc = formMetacellTags<Pt>(vol_d, pd, md, g, nm, 0, 1, 32);
		auto h = fetch(mc, nm);
		if (nm != 8u * 4u * 2u || h[5].id != 5u || h[5].dim1_val > h[5].dim2_val)
			failures++;
		cudaFree(vol_d);
	}
	cudaFree(pts_d);
	if (failures) {
		std::printf("FACADE FAILED (%d)\n", failures);
		return 1;
	}
	std::printf("FACADE OK\n");
	return 0;
}
