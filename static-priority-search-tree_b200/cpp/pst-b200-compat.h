// PointStruct and the StaticPrioritySearchTree base with the reference's layout and
// interface, for code that does not include the reference's own headers.  The
// include guards are the reference's (POINT_STRUCT_H, STATIC_PRIORITY_SEARCH_TREE_H),
// so when its helpers/point-struct.h or pst/static-priority-search-tree.h come
// first, those definitions are used and these are skipped.
#ifndef PST_B200_COMPAT_H
#define PST_B200_COMPAT_H

#include <cstddef>
#include <ostream>
#include <type_traits>

#ifndef POINT_STRUCT_H
#define POINT_STRUCT_H

template <typename T, typename IDType, size_t num_IDs>
struct PointStruct;

// Record layouts of helpers/point-struct.h:25-33 and :106-117.
template <typename T>
struct PointStruct<T, void, 0> {
	static_assert(std::is_arithmetic<T>::value, "Input type T not of arithmetic type");
	T dim1_val;
	T dim2_val;
	PointStruct() : dim1_val(0), dim2_val(0) {}
	PointStruct(T d1, T d2) : dim1_val(d1), dim2_val(d2) {}
	void print(std::ostream &os) const { os << '(' << dim1_val << ", " << dim2_val << ')'; }
	bool operator==(const PointStruct &o) const { return dim1_val == o.dim1_val && dim2_val == o.dim2_val; }
};

template <typename T, typename IDType>
struct PointStruct<T, IDType, 1> {
	static_assert(std::is_arithmetic<T>::value, "Input type T not of arithmetic type");
	T dim1_val;
	T dim2_val;
	IDType id;
	PointStruct() : dim1_val(0), dim2_val(0), id(0) {}
	PointStruct(T d1, T d2, IDType i) : dim1_val(d1), dim2_val(d2), id(i) {}
	void print(std::ostream &os) const { os << '(' << dim1_val << ", " << dim2_val << "; " << id << ')'; }
	bool operator==(const PointStruct &o) const
	{
		return dim1_val == o.dim1_val && dim2_val == o.dim2_val && id == o.id;
	}
};

template <typename T, size_t num_IDs, typename IDType>
std::ostream &operator<<(std::ostream &os, const PointStruct<T, IDType, num_IDs> &p)
{
	p.print(os);
	return os;
}

#endif  // POINT_STRUCT_H

#ifndef STATIC_PRIORITY_SEARCH_TREE_H
#define STATIC_PRIORITY_SEARCH_TREE_H

// pst/static-priority-search-tree.h:9-28: virtual print and operator<<.
template <typename T, template <typename, typename, size_t> class PointStructTemplate, typename IDType, size_t num_IDs>
class StaticPrioritySearchTree
{
  public:
	virtual ~StaticPrioritySearchTree() {}
	virtual void print(std::ostream &os) const = 0;
};

template <typename T, template <typename, typename, size_t> class PointStructTemplate, typename IDType, size_t num_IDs>
std::ostream &operator<<(std::ostream &os, const StaticPrioritySearchTree<T, PointStructTemplate, IDType, num_IDs> &t)
{
	t.print(os);
	return os;
}

#endif  // STATIC_PRIORITY_SEARCH_TREE_H

#endif
