// Host-only harness that compiles the reference's own StaticPSTCPUIter and
// StaticPSTCPURecur, unmodified, from their sources (pst/static-pst-cpu-iter.h,
// pst/static-pst-cpu-recur.h and the headers they include) into
// oracle/_ref/libpstref.so.  The recursive tree is a second, independent CPU
// implementation of the same searches in the reference; it cross-checks the first.  TEST INFRASTRUCTURE ONLY: it pins the oracle, makes
// the golden fixtures, and is the timed CPU baseline ("reference" kind) of the
// benchmark.  Nothing in the product links it.
//
// The tree's storage members are private in the reference; the harness reads them
// (to compare whole trees bit for bit) by compiling the class with `private`
// mapped to `public` in this translation unit only.  Standard headers are
// included first so that the mapping only touches the reference's own classes.
#include <algorithm>
#include <cassert>    // pst/static-pst-cpu-iter-populate-tree.tpp:58 uses assert without including it
#include <concepts>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <ostream>
#include <stack>
#include <stdexcept>
#include <string>
#include <type_traits>

#define private public
#include "point-struct.h"
#include "static-pst-cpu-iter.h"
#include "static-pst-cpu-recur.h"
#undef private

namespace {

enum { REF_F32 = 0, REF_F64 = 1, REF_I32 = 2 };
enum { REF_Q_THREE = 0, REF_Q_LEFT = 1, REF_Q_RIGHT = 2 };

struct Handle {
	int dtype;
	int has_id;
	void *tree;
	int recur;  // StaticPSTCPURecur instead of StaticPSTCPUIter
};

template <typename T, int HAS_ID>
struct Types;
template <typename T>
struct Types<T, 1> {
	using Pt = PointStruct<T, uint32_t, 1>;
	using Tree = StaticPSTCPUIter<T, PointStruct, uint32_t, 1>;
	using Recur = StaticPSTCPURecur<T, PointStruct, uint32_t, 1>;
};
template <typename T>
struct Types<T, 0> {
	using Pt = PointStruct<T, void, 0>;
	using Tree = StaticPSTCPUIter<T, PointStruct, void, 0>;
	using Recur = StaticPSTCPURecur<T, PointStruct, void, 0>;
};

template <typename T, int HAS_ID, bool RECUR = false>
void *build(const void *pts, uint64_t n)
{
	using Tr = std::conditional_t<RECUR, typename Types<T, HAS_ID>::Recur, typename Types<T, HAS_ID>::Tree>;
	using Pt = typename Types<T, HAS_ID>::Pt;
	// The constructor only reads the array, but its signature takes a non-const pointer
	return new Tr(const_cast<Pt *>(static_cast<const Pt *>(pts)), n);
}

template <typename T, int HAS_ID, bool RECUR = false>
void destroy(void *t)
{
	using Tr = std::conditional_t<RECUR, typename Types<T, HAS_ID>::Recur, typename Types<T, HAS_ID>::Tree>;
	delete static_cast<Tr *>(t);
}

template <typename T, int HAS_ID>
uint64_t slots(void *t)
{
	return static_cast<typename Types<T, HAS_ID>::Tree *>(t)->num_elem_slots;
}

// Copies the tree's single allocation out field by field through the reference's
// own accessors (pst/static-pst-cpu-iter.h:130-153).
template <typename T, int HAS_ID>
void export_tree(void *tp, T *dim1, T *dim2, T *med, uint32_t *ids, uint8_t *bitcodes)
{
	using Tr = typename Types<T, HAS_ID>::Tree;
	Tr *t = static_cast<Tr *>(tp);
	const size_t S = t->num_elem_slots;
	if (S == 0)
		return;
	std::memcpy(dim1, Tr::getDim1ValsRoot(t->root, S), S * sizeof(T));
	std::memcpy(dim2, Tr::getDim2ValsRoot(t->root, S), S * sizeof(T));
	std::memcpy(med, Tr::getMedDim1ValsRoot(t->root, S), S * sizeof(T));
	if constexpr (HAS_ID)
		std::memcpy(ids, Tr::getIDsRoot(t->root, S), S * sizeof(uint32_t));
	std::memcpy(bitcodes, Tr::getBitcodesRoot(t->root, S), S);
}

// Runs one reference search.  ret_points = 0 returns ids (id trees only), 1 returns
// PointStruct records.  The result array is allocated by the reference (new[]),
// copied out (up to cap records) and freed here.  Returns the count, or -1.
template <typename T, int HAS_ID, bool RECUR = false>
int64_t search(void *tp, int kind, T min1, T max1, T min2, int ret_points, void *out, uint64_t cap)
{
	using Tr = std::conditional_t<RECUR, typename Types<T, HAS_ID>::Recur, typename Types<T, HAS_ID>::Tree>;
	using Pt = typename Types<T, HAS_ID>::Pt;
	Tr *t = static_cast<Tr *>(tp);
	size_t cnt = 0;
	auto run = [&](auto *dummy) -> int64_t {
		using R = std::remove_pointer_t<decltype(dummy)>;
		R *res = nullptr;
		if (kind == REF_Q_THREE)
			t->template threeSidedSearch<R>(cnt, res, min1, max1, min2);
		else if (kind == REF_Q_LEFT)
			t->template twoSidedLeftSearch<R>(cnt, res, max1, min2);
		else
			t->template twoSidedRightSearch<R>(cnt, res, min1, min2);
		if (out && res)
			std::memcpy(out, res, std::min<size_t>(cnt, cap) * sizeof(R));
		delete[] res;
		return static_cast<int64_t>(cnt);
	};
	if constexpr (HAS_ID) {
		if (!ret_points)
			return run(static_cast<uint32_t *>(nullptr));
	}
	return run(static_cast<Pt *>(nullptr));
}

template <typename F>
auto dispatch(int dtype, int has_id, F &&f)
{
	if (dtype == REF_F32)
		return has_id ? f.template operator()<float, 1>() : f.template operator()<float, 0>();
	if (dtype == REF_F64)
		return has_id ? f.template operator()<double, 1>() : f.template operator()<double, 0>();
	return has_id ? f.template operator()<int32_t, 1>() : f.template operator()<int32_t, 0>();
}

template <typename T>
T as(const void *p)
{
	T v;
	std::memcpy(&v, p, sizeof(T));
	return v;
}

}  // namespace

extern "C" {

// Builds a StaticPSTCPUIter over `n` PointStruct records at `pts` (host memory).
void *ref_build(int dtype, int has_id, const void *pts, uint64_t n)
{
	try {
		Handle *h = new Handle{dtype, has_id, nullptr, 0};
		h->tree = dispatch(dtype, has_id, [&]<typename T, int I>() { return build<T, I>(pts, n); });
		return h;
	} catch (...) {
		return nullptr;
	}
}

// Builds a StaticPSTCPURecur (searches only: ref_search; no export).
void *ref_build_recur(int dtype, int has_id, const void *pts, uint64_t n)
{
	try {
		Handle *h = new Handle{dtype, has_id, nullptr, 1};
		h->tree = dispatch(dtype, has_id, [&]<typename T, int I>() { return build<T, I, true>(pts, n); });
		return h;
	} catch (...) {
		return nullptr;
	}
}

void ref_destroy(void *hp)
{
	if (!hp)
		return;
	Handle *h = static_cast<Handle *>(hp);
	dispatch(h->dtype, h->has_id, [&]<typename T, int I>() {
		if (h->recur)
			destroy<T, I, true>(h->tree);
		else
			destroy<T, I>(h->tree);
		return 0;
	});
	delete h;
}

uint64_t ref_num_slots(void *hp)
{
	Handle *h = static_cast<Handle *>(hp);
	return dispatch(h->dtype, h->has_id, [&]<typename T, int I>() { return slots<T, I>(h->tree); });
}

void ref_export(void *hp, void *dim1, void *dim2, void *med, uint32_t *ids, uint8_t *bitcodes)
{
	Handle *h = static_cast<Handle *>(hp);
	dispatch(h->dtype, h->has_id, [&]<typename T, int I>() {
		export_tree<T, I>(h->tree, static_cast<T *>(dim1), static_cast<T *>(dim2),
		                  static_cast<T *>(med), ids, bitcodes);
		return 0;
	});
}

// Bounds are passed by address in the tree's value type.
int64_t ref_search(void *hp, int kind, const void *min1, const void *max1, const void *min2,
                   int ret_points, void *out, uint64_t cap)
{
	Handle *h = static_cast<Handle *>(hp);
	try {
		return dispatch(h->dtype, h->has_id, [&]<typename T, int I>() {
			if (h->recur)
				return search<T, I, true>(h->tree, kind, as<T>(min1), as<T>(max1), as<T>(min2), ret_points, out, cap);
			return search<T, I>(h->tree, kind, as<T>(min1), as<T>(max1), as<T>(min2), ret_points, out, cap);
		});
	} catch (...) {
		return -1;
	}
}

}  // extern "C"
