/*
 * CPU oracle for the static priority search tree path.  TEST INFRASTRUCTURE ONLY:
 * the parity tests, the smoke check and the CPU-baseline leg of the benchmark
 * use it as the checker.  No product code path links or calls it.
 *
 * Parity status: pinned.  The tree, the searches and the interval scan are
 * checked against the reference implementation itself (StaticPSTCPUIter compiled
 * unmodified from its own sources into oracle/_ref/libpstref.so) by
 * tests/test_oracle_pin.py, and against golden fixtures produced by that compiled
 * reference (tests/golden/make_golden.py).  Metacell formation is checked against
 * the reference's own metacell kernel (compiled from its sources into
 * oracle/_ref/libmcref.so by ref_metacells.cu) in tests/test_gpu_metacell_pin.py,
 * on the sizes that kernel handles (it needs a GPU to run).  The many-query brute
 * force (orc_brute_multi) is checked against the one-query brute force in
 * tests/test_oracle_brute_multi.py.
 *
 * Restated from the reference (paths relative to the reference project):
 *   - point total order          helpers/point-struct.h:62-92, :154-188
 *   - index sorts                pst/static-pst-cpu-iter.tpp:78-116
 *   - explicit-stack population  pst/static-pst-cpu-iter-populate-tree.tpp:11-114
 *   - binarySearch               pst/static-pst-cpu-iter.tpp:793-818
 *   - constructNode              pst/static-pst-cpu-iter.tpp:491-598
 *   - searches + delegation      pst/static-pst-cpu-iter.tpp:204-486, :602-735
 *   - tree memory layout         pst/static-pst-cpu-iter.h:130-153, .tpp:740-789
 *   - interval parallel search   interval-parallel-search/interval-parallel-search.h:91-116
 *   - metacell formation         helpers/isosurface-data-processing.h:23-36,
 *                                helpers/isosurface-data-processing.tu:9-127, :181-212
 *
 * Points are passed as the reference's PointStruct records:
 *   with id:    { T dim1; T dim2; uint32_t id; }   (natural C alignment/padding)
 *   without id: { T dim1; T dim2; }
 * The "address" tiebreak of the reference (comparisonTiebreaker compares
 * this-pointers inside one contiguous array) is the input index here.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { ORC_F32 = 0, ORC_F64 = 1, ORC_I32 = 2 };
enum { ORC_Q_THREE = 0, ORC_Q_LEFT = 1, ORC_Q_RIGHT = 2 };
/* Search codes, pst/static-pst-cpu-iter.h:206-212 */
enum { SC_REPORT_ABOVE = 0, SC_LEFT = 1, SC_RIGHT = 2, SC_THREE = 3 };
/* Child-presence bitcodes, pst/cpu-iter-tree-node.h:42-46 */
enum { HAS_LEFT = 0x2, HAS_RIGHT = 0x1 };

/* Number of slots of the implicit tree: minPowerOf2GreaterThan(n) - 1
 * (helpers/power-of-2-functions.h:51-61, :103-106). */
uint64_t orc_num_slots(uint64_t n)
{
	if (n == 0)
		return 0;
	unsigned e = 0;
	while ((n >> e) != 0)
		e++;
	return (1ull << e) - 1;
}

/* Level parity used to alternate the primary/secondary dim2 arrays:
 * expOfMinPowerOf2GreaterThan(node + 1) % 2
 * (pst/static-pst-cpu-iter-populate-tree.tpp:40). */
static unsigned exp_min_pow2_gt(uint64_t v)
{
	unsigned e = 0;
	while ((v >> e) != 0)
		e++;
	return e;
}

typedef struct {
	size_t *a;	/* index stack storage */
	size_t top, cap;
} stk_t;

static int stk_push(stk_t *s, size_t v)
{
	if (s->top == s->cap) {
		size_t nc = s->cap ? 2 * s->cap : 64;
		size_t *na = (size_t *) realloc(s->a, nc * sizeof(size_t));
		if (!na)
			return -1;
		s->a = na;
		s->cap = nc;
	}
	s->a[s->top++] = v;
	return 0;
}

/*
 * The whole oracle is generated once per value type by ORACLE_DEFINE.
 * Stride/offsets describe the point record layout so that one body serves the
 * id and id-less variants.
 */
#define ORACLE_DEFINE(SFX, T)                                                                 \
                                                                                               \
typedef struct {                                                                               \
	const unsigned char *base;                                                                 \
	size_t stride;                                                                             \
	size_t id_off;                                                                             \
	int has_id;                                                                                \
} pts_##SFX;                                                                                   \
                                                                                               \
static inline T d1_##SFX(const pts_##SFX *p, size_t i)                                         \
{ T v; memcpy(&v, p->base + i * p->stride, sizeof(T)); return v; }                             \
static inline T d2_##SFX(const pts_##SFX *p, size_t i)                                         \
{ T v; memcpy(&v, p->base + i * p->stride + sizeof(T), sizeof(T)); return v; }                \
static inline uint32_t id_##SFX(const pts_##SFX *p, size_t i)                                  \
{ uint32_t v = 0; if (p->has_id) memcpy(&v, p->base + i * p->stride + p->id_off, 4); return v; } \
                                                                                               \
/* comparisonTiebreaker, helpers/point-struct.h:89-92 (no id) and :181-188 (id):              \
 * id first when present, then the position in the contiguous input array. */                 \
static inline int tie_##SFX(const pts_##SFX *p, size_t i, size_t j)                            \
{                                                                                              \
	if (p->has_id) {                                                                           \
		uint32_t a = id_##SFX(p, i), b = id_##SFX(p, j);                                       \
		if (a != b)                                                                            \
			return a < b ? -1 : 1;                                                             \
	}                                                                                          \
	return i == j ? 0 : (i < j ? -1 : 1);                                                      \
}                                                                                              \
/* compareDim1 / compareDim2, helpers/point-struct.h:62-81, :154-173 */                        \
static inline int cmp1_##SFX(const pts_##SFX *p, size_t i, size_t j)                           \
{                                                                                              \
	T a = d1_##SFX(p, i), b = d1_##SFX(p, j);                                                  \
	if (a != b)                                                                                \
		return a < b ? -1 : 1;                                                                 \
	return tie_##SFX(p, i, j);                                                                 \
}                                                                                              \
static inline int cmp2_##SFX(const pts_##SFX *p, size_t i, size_t j)                           \
{                                                                                              \
	T a = d2_##SFX(p, i), b = d2_##SFX(p, j);                                                  \
	if (a != b)                                                                                \
		return a < b ? -1 : 1;                                                                 \
	return tie_##SFX(p, i, j);                                                                 \
}                                                                                              \
                                                                                               \
/* Stable merge sort of an index array; the comparators are total orders, so                 \
 * any correct sort yields the same permutation as the reference's std::sort. */             \
static void msort_##SFX(const pts_##SFX *p, size_t *a, size_t *tmp, size_t n, int dim, int desc) \
{                                                                                              \
	for (size_t w = 1; w < n; w <<= 1) {                                                       \
		for (size_t lo = 0; lo < n; lo += 2 * w) {                                             \
			size_t mid = lo + w < n ? lo + w : n;                                              \
			size_t hi = lo + 2 * w < n ? lo + 2 * w : n;                                       \
			size_t i = lo, j = mid, k = lo;                                                    \
			while (i < mid && j < hi) {                                                        \
				int c = dim == 1 ? cmp1_##SFX(p, a[j], a[i]) : cmp2_##SFX(p, a[j], a[i]);      \
				if (desc)                                                                      \
					c = -c;                                                                    \
				tmp[k++] = c < 0 ? a[j++] : a[i++];                                            \
			}                                                                                  \
			while (i < mid)                                                                    \
				tmp[k++] = a[i++];                                                             \
			while (j < hi)                                                                     \
				tmp[k++] = a[j++];                                                             \
		}                                                                                      \
		memcpy(a, tmp, n * sizeof(size_t));                                                    \
	}                                                                                          \
}                                                                                              \
                                                                                               \
/* binarySearch, pst/static-pst-cpu-iter.tpp:793-818: the position of point e in the        \
 * dim1-ordered index subarray [lo, lo + num). */                                             \
static long long bsearch_##SFX(const pts_##SFX *p, const size_t *d1a, size_t e,              \
                               size_t lo, size_t num)                                          \
{                                                                                              \
	size_t hi = lo + num;                                                                      \
	while (lo < hi) {                                                                          \
		size_t mid = (lo + hi) / 2;                                                            \
		if (d1a[mid] == e)                                                                     \
			return (long long) mid;                                                            \
		else if (cmp1_##SFX(p, e, d1a[mid]) < 0)                                               \
			hi = mid;                                                                          \
		else                                                                                   \
			lo = mid + 1;                                                                      \
	}                                                                                          \
	return -1;                                                                                 \
}                                                                                              \
                                                                                               \
/* Builds the tree into separate field arrays laid out exactly like the reference's         \
 * single allocation (dim1, dim2, med, id, bitcode; slot s = heap index, root 0).            \
 * Arrays must hold orc_num_slots(n) entries and be zeroed by the caller (the reference       \
 * value-initialises its allocation, pst/static-pst-cpu-iter.tpp:38,44).                      \
 * Returns 0 on success, -1 on allocation failure, -2 on an internal inconsistency. */       \
int orc_build_##SFX(const void *pts, size_t stride, size_t id_off, int has_id, uint64_t n,    \
                    T *dim1, T *dim2, T *med, uint32_t *ids, uint8_t *bitcodes)               \
{                                                                                              \
	if (n == 0)                                                                                \
		return 0;                                                                              \
	pts_##SFX P = { (const unsigned char *) pts, stride, id_off, has_id };                    \
	size_t *d1a = (size_t *) malloc(n * sizeof(size_t));                                       \
	size_t *d2a = (size_t *) malloc(n * sizeof(size_t));                                       \
	size_t *d2b = (size_t *) malloc(n * sizeof(size_t));                                       \
	stk_t st = {0}, sn = {0}, sh = {0};                                                        \
	int rc = 0;                                                                                \
	if (!d1a || !d2a || !d2b) { rc = -1; goto done; }                                          \
	/* pst/static-pst-cpu-iter.tpp:78-116: iota, dim1 ascending, dim2 descending */           \
	for (size_t i = 0; i < n; i++)                                                             \
		d1a[i] = d2a[i] = i;                                                                   \
	msort_##SFX(&P, d1a, d2b, n, 1, 0);                                                        \
	msort_##SFX(&P, d2a, d2b, n, 2, 1);                                                        \
	/* populateTree, pst/static-pst-cpu-iter-populate-tree.tpp:17-113 */                      \
	if (stk_push(&st, 0) || stk_push(&sn, n) || stk_push(&sh, 0)) { rc = -1; goto done; }     \
	while (st.top) {                                                                           \
		size_t start = st.a[st.top - 1], num = sn.a[sn.top - 1], node = sh.a[sh.top - 1];      \
		size_t *prim, *sec;                                                                    \
		if (exp_min_pow2_gt(node + 1) % 2) { prim = d2a; sec = d2b; }                          \
		else { prim = d2b; sec = d2a; }                                                        \
		long long found = bsearch_##SFX(&P, d1a, prim[start], start, num);                     \
		if (found < 0) { rc = -2; goto done; }                                                 \
		size_t pmax = (size_t) found;                                                          \
		/* constructNode, pst/static-pst-cpu-iter.tpp:508-597 */                              \
		size_t medi, nleft, nright;                                                            \
		if (num == 1) { medi = start; nleft = 0; nright = 0; }                                 \
		else if (pmax < start + num / 2) {                                                     \
			medi = start + num / 2;                                                            \
			nleft = medi - start;                                                              \
			nright = start + num - medi - 1;                                                   \
		} else {                                                                               \
			medi = start + num / 2 - 1;                                                        \
			nleft = medi - start + 1;                                                          \
			nright = start + num - medi - 2;                                                   \
		}                                                                                      \
		size_t top = prim[start];                                                              \
		size_t medpt = d1a[medi];                                                              \
		dim1[node] = d1_##SFX(&P, top);                                                        \
		dim2[node] = d2_##SFX(&P, top);                                                        \
		med[node] = d1_##SFX(&P, medpt);                                                       \
		if (has_id && ids)                                                                     \
			ids[node] = id_##SFX(&P, top);                                                     \
		if (nleft > 0) {                                                                       \
			bitcodes[node] |= HAS_LEFT;                                                        \
			if (pmax < medi)                                                                   \
				for (size_t i = pmax; i < medi; i++)                                           \
					d1a[i] = d1a[i + 1];                                                       \
		}                                                                                      \
		if (nright > 0) {                                                                      \
			bitcodes[node] |= HAS_RIGHT;                                                       \
			if (pmax > medi)                                                                   \
				for (size_t i = pmax; i < start + num - 1; i++)                                \
					d1a[i] = d1a[i + 1];                                                       \
		}                                                                                      \
		size_t rstart = medi + 1;                                                              \
		if (bitcodes[node] & (HAS_LEFT | HAS_RIGHT)) {                                         \
			size_t li = start, ri = rstart;                                                    \
			for (size_t i = start + 1; i < start + num; i++) {                                 \
				if (cmp1_##SFX(&P, prim[i], medpt) <= 0)                                       \
					sec[li++] = prim[i];                                                       \
				else                                                                           \
					sec[ri++] = prim[i];                                                       \
			}                                                                                  \
		}                                                                                      \
		st.top--; sn.top--; sh.top--;                                                          \
		if (nright > 0)                                                                        \
			if (stk_push(&sh, 2 * node + 2) || stk_push(&st, rstart) || stk_push(&sn, nright)) \
				{ rc = -1; goto done; }                                                        \
		if (nleft > 0)                                                                         \
			if (stk_push(&sh, 2 * node + 1) || stk_push(&st, start) || stk_push(&sn, nleft))   \
				{ rc = -1; goto done; }                                                        \
	}                                                                                          \
done:                                                                                          \
	free(d1a); free(d2a); free(d2b);                                                           \
	free(st.a); free(sn.a); free(sh.a);                                                        \
	return rc;                                                                                 \
}                                                                                              \
                                                                                               \
/* Searches, pst/static-pst-cpu-iter.tpp:204-486 with the delegation helpers of :602-735.     \
 * Writes reported heap slots to out_slots (capacity n) in the reference's report order      \
 * and returns their number.  kind selects the query; unused bounds are ignored. */          \
int64_t orc_search_##SFX(const T *dim1, const T *dim2, const T *med, const uint8_t *bitcodes, \
                         uint64_t n, int kind, T min1, T max1, T min2, uint64_t *out_slots)    \
{                                                                                              \
	if (n == 0)                                                                                \
		return 0;                                                                              \
	stk_t si = {0}, sc = {0};                                                                  \
	int64_t cnt = 0;                                                                           \
	int code0 = kind == ORC_Q_THREE ? SC_THREE : kind == ORC_Q_LEFT ? SC_LEFT : SC_RIGHT;       \
	if (stk_push(&si, 0) || stk_push(&sc, (size_t) code0)) { cnt = -1; goto sdone; }           \
	while (si.top) {                                                                           \
		size_t s = si.a[--si.top];                                                             \
		int code = (int) sc.a[--sc.top];                                                       \
		T v1 = dim1[s], v2 = dim2[s], vm = med[s];                                             \
		uint8_t bc = bitcodes[s];                                                              \
		if (!(min2 <= v2))                                                                     \
			continue;                                                                          \
		/* Each search function tests its own query's predicate at every node,                \
		 * whatever the node's search code (:250-251, :358, :449). */                         \
		int rep = kind == ORC_Q_THREE ? (min1 <= v1 && v1 <= max1)                             \
		        : kind == ORC_Q_LEFT ? (v1 <= max1) : (v1 >= min1);                            \
		if (rep)                                                                               \
			out_slots[cnt++] = s;                                                              \
		if (!(bc & (HAS_LEFT | HAS_RIGHT)))                                                    \
			continue;                                                                          \
		size_t l = 2 * s + 1, r = 2 * s + 2;                                                   \
		int e = 0;                                                                             \
		if (code == SC_THREE) {                                                                \
			if (min1 <= vm && vm <= max1) {                                                    \
				if (bc & HAS_LEFT) e |= stk_push(&si, l) | stk_push(&sc, SC_RIGHT);             \
				if (bc & HAS_RIGHT) e |= stk_push(&si, r) | stk_push(&sc, SC_LEFT);             \
			} else if (max1 < vm && (bc & HAS_LEFT))                                           \
				e |= stk_push(&si, l) | stk_push(&sc, SC_THREE);                               \
			else if (vm < min1 && (bc & HAS_RIGHT))                                            \
				e |= stk_push(&si, r) | stk_push(&sc, SC_THREE);                               \
		} else if (code == SC_LEFT) {                                                          \
			if (vm <= max1) {                                                                  \
				if (bc & HAS_LEFT) e |= stk_push(&si, l) | stk_push(&sc, SC_REPORT_ABOVE);      \
				if (bc & HAS_RIGHT) e |= stk_push(&si, r) | stk_push(&sc, SC_LEFT);             \
			} else if (bc & HAS_LEFT)                                                          \
				e |= stk_push(&si, l) | stk_push(&sc, SC_LEFT);                                \
		} else if (code == SC_RIGHT) {                                                         \
			if (vm >= min1) {                                                                  \
				if (bc & HAS_LEFT) e |= stk_push(&si, l) | stk_push(&sc, SC_RIGHT);             \
				if (bc & HAS_RIGHT) e |= stk_push(&si, r) | stk_push(&sc, SC_REPORT_ABOVE);     \
			} else if (bc & HAS_RIGHT)                                                         \
				e |= stk_push(&si, r) | stk_push(&sc, SC_RIGHT);                               \
		} else {                                                                               \
			if (bc & HAS_LEFT) e |= stk_push(&si, l) | stk_push(&sc, SC_REPORT_ABOVE);          \
			if (bc & HAS_RIGHT) e |= stk_push(&si, r) | stk_push(&sc, SC_REPORT_ABOVE);         \
		}                                                                                      \
		if (e) { cnt = -1; goto sdone; }                                                       \
	}                                                                                          \
sdone:                                                                                         \
	free(si.a); free(sc.a);                                                                    \
	return cnt;                                                                                \
}                                                                                              \
                                                                                               \
/* Brute-force predicate of the three query kinds (the definitions used by                  \
 * pst/static-pst-cpu-iter.tpp:247-251, :355-358, :446-449).  Writes input indices. */       \
int64_t orc_brute_##SFX(const void *pts, size_t stride, uint64_t n, int kind,                 \
                        T min1, T max1, T min2, uint64_t *out_idx)                             \
{                                                                                              \
	pts_##SFX P = { (const unsigned char *) pts, stride, 0, 0 };                               \
	int64_t cnt = 0;                                                                           \
	for (uint64_t i = 0; i < n; i++) {                                                         \
		T v1 = d1_##SFX(&P, i), v2 = d2_##SFX(&P, i);                                          \
		if (!(min2 <= v2))                                                                     \
			continue;                                                                          \
		int ok = kind == ORC_Q_THREE ? (min1 <= v1 && v1 <= max1)                              \
		       : kind == ORC_Q_LEFT ? (v1 <= max1) : (v1 >= min1);                             \
		if (ok)                                                                                \
			out_idx[cnt++] = i;                                                                \
	}                                                                                          \
	return cnt;                                                                                \
}                                                                                              \
                                                                                               \
/* Interval parallel search predicate dim1 <= v <= dim2,                                     \
 * interval-parallel-search/interval-parallel-search.h:94-96.  Writes input indices. */      \
int64_t orc_ips_##SFX(const void *pts, size_t stride, uint64_t n, T v, uint64_t *out_idx)     \
{                                                                                              \
	pts_##SFX P = { (const unsigned char *) pts, stride, 0, 0 };                               \
	int64_t cnt = 0;                                                                           \
	for (uint64_t i = 0; i < n; i++)                                                           \
		if (d1_##SFX(&P, i) <= v && v <= d2_##SFX(&P, i))                                      \
			out_idx[cnt++] = i;                                                                \
	return cnt;                                                                                \
}                                                                                              \
                                                                                               \
/* Metacell formation: calcNumMetacells (helpers/isosurface-data-processing.h:23-36) and     \
 * the per-metacell min/max over the vertices of the metacell's valid voxels                 \
 * (getVoxelMinMax + the block reduction of formMetacellTagsGlobal,                          \
 * helpers/isosurface-data-processing.tu:9-127, :181-212).  Metacell (mx,my,mz) covers        \
 * voxels [m*mc, min(m*mc+mc, P-1)) per axis, i.e. vertices [m*mc, min(m*mc+mc, P-1)].        \
 * id = lineariseID(mx, my, mz) = mx + (my + mz*My)*Mx (helpers/linearise-id.h:13-19).        \
 * Output arrays are indexed by metacell id.  Returns the number of metacells. */            \
int64_t orc_metacells_##SFX(const T *vol, uint32_t px, uint32_t py, uint32_t pz,              \
                            uint32_t mcx, uint32_t mcy, uint32_t mcz,                          \
                            T *out_min, T *out_max, uint32_t *out_id)                          \
{                                                                                              \
	if (px < 2 || py < 2 || pz < 2 || !mcx || !mcy || !mcz)                                    \
		return 0;                                                                              \
	uint64_t Mx = (px - 1 + mcx - 1) / mcx, My = (py - 1 + mcy - 1) / mcy;                     \
	uint64_t Mz = (pz - 1 + mcz - 1) / mcz;                                                    \
	for (uint64_t mz = 0; mz < Mz; mz++)                                                       \
	for (uint64_t my = 0; my < My; my++)                                                       \
	for (uint64_t mx = 0; mx < Mx; mx++) {                                                     \
		uint64_t x0 = mx * mcx, y0 = my * mcy, z0 = mz * mcz;                                  \
		uint64_t x1 = x0 + mcx < px - 1 ? x0 + mcx : px - 1;                                   \
		uint64_t y1 = y0 + mcy < py - 1 ? y0 + mcy : py - 1;                                   \
		uint64_t z1 = z0 + mcz < pz - 1 ? z0 + mcz : pz - 1;                                   \
		T lo = vol[x0 + (y0 + z0 * py) * px], hi = lo;                                         \
		for (uint64_t z = z0; z <= z1; z++)                                                    \
		for (uint64_t y = y0; y <= y1; y++)                                                    \
		for (uint64_t x = x0; x <= x1; x++) {                                                  \
			T v = vol[x + (y + z * py) * px];                                                  \
			if (v < lo) lo = v;                                                                \
			if (v > hi) hi = v;                                                                \
		}                                                                                      \
		uint64_t id = mx + (my + mz * My) * Mx;                                                \
		out_min[id] = lo;                                                                      \
		out_max[id] = hi;                                                                      \
		if (out_id)                                                                            \
			out_id[id] = (uint32_t) id;                                                        \
	}                                                                                          \
	return (int64_t) (Mx * My * Mz);                                                           \
}

ORACLE_DEFINE(f32, float)
ORACLE_DEFINE(f64, double)
ORACLE_DEFINE(i32, int32_t)

/*
 * Brute force of many queries over one point set at once (the same predicates as
 * orc_brute_*), for checking large trees: the points are read once per pass
 * instead of once per query.  Threads take contiguous point ranges; pass 1 counts
 * each (thread, query) pair over blocks of BRUTE_BLOCK points, pass 2 writes the
 * input indices of each query's hits, in index order, at out_off[q].
 * out_off receives nq + 1 offsets (exclusive scan of the per-query counts);
 * out_idx (may be NULL: counts only) must hold out_off[nq] entries.
 * Returns the total number of hits, or -1 when a thread or buffer cannot be had.
 */
#define BRUTE_BLOCK 2048

#define BRUTE_MULTI_DEFINE(SFX, T)                                                             \
typedef struct {                                                                               \
	const unsigned char *pts; size_t stride; uint64_t lo, hi;                                  \
	uint32_t nq; const int32_t *kinds; const T *min1, *max1, *min2;                           \
	uint64_t *cnt;        /* nq counts of this thread (pass 1) */                               \
	uint64_t *pos;        /* nq write positions of this thread (pass 2) */                      \
	uint64_t *out_idx;                                                                         \
	int pass;                                                                                  \
} bm_##SFX;                                                                                    \
                                                                                               \
static void *bm_run_##SFX(void *arg)                                                           \
{                                                                                              \
	bm_##SFX *a = (bm_##SFX *) arg;                                                            \
	T v1[BRUTE_BLOCK], v2[BRUTE_BLOCK];                                                        \
	for (uint64_t b = a->lo; b < a->hi; b += BRUTE_BLOCK) {                                    \
		const uint64_t m = a->hi - b < BRUTE_BLOCK ? a->hi - b : BRUTE_BLOCK;                  \
		for (uint64_t i = 0; i < m; i++) {                                                     \
			memcpy(&v1[i], a->pts + (b + i) * a->stride, sizeof(T));                           \
			memcpy(&v2[i], a->pts + (b + i) * a->stride + sizeof(T), sizeof(T));               \
		}                                                                                      \
		for (uint32_t q = 0; q < a->nq; q++) {                                                 \
			const int k = a->kinds[q];                                                         \
			const T m2 = a->min2[q];                                                           \
			const int use_lo = k != ORC_Q_LEFT, use_hi = k != ORC_Q_RIGHT;                     \
			if (a->pass == 1) {                                                                \
				uint64_t c = 0;                                                                \
				for (uint64_t i = 0; i < m; i++)                                               \
					c += (m2 <= v2[i]) & (!use_lo | (a->min1[q] <= v1[i]))                     \
					     & (!use_hi | (v1[i] <= a->max1[q]));                                  \
				a->cnt[q] += c;                                                                \
			} else {                                                                           \
				uint64_t w = a->pos[q];                                                        \
				for (uint64_t i = 0; i < m; i++)                                               \
					if ((m2 <= v2[i]) & (!use_lo | (a->min1[q] <= v1[i]))                      \
					    & (!use_hi | (v1[i] <= a->max1[q])))                                   \
						a->out_idx[w++] = b + i;                                               \
				a->pos[q] = w;                                                                 \
			}                                                                                  \
		}                                                                                      \
	}                                                                                          \
	return NULL;                                                                               \
}                                                                                              \
                                                                                               \
int64_t orc_brute_multi_##SFX(const void *pts, size_t stride, uint64_t n, uint32_t nq,        \
                              const int32_t *kinds, const T *min1, const T *max1,              \
                              const T *min2, int threads, uint64_t *out_off,                   \
                              uint64_t *out_idx)                                               \
{                                                                                              \
	if (threads < 1) threads = 1;                                                              \
	if ((uint64_t) threads > n / BRUTE_BLOCK + 1) threads = (int) (n / BRUTE_BLOCK + 1);       \
	bm_##SFX *job = calloc((size_t) threads, sizeof(bm_##SFX));                                \
	pthread_t *th = calloc((size_t) threads, sizeof(pthread_t));                               \
	uint64_t *cnt = calloc((size_t) threads * (nq ? nq : 1), sizeof(uint64_t));                \
	uint64_t *pos = calloc((size_t) threads * (nq ? nq : 1), sizeof(uint64_t));                \
	int64_t total = -1;                                                                        \
	if (!job || !th || !cnt || !pos)                                                           \
		goto done;                                                                             \
	const uint64_t per = (n + (uint64_t) threads - 1) / (uint64_t) threads;                    \
	for (int t = 0; t < threads; t++) {                                                        \
		uint64_t lo = per * (uint64_t) t, hi = lo + per;                                       \
		if (lo > n) lo = n;                                                                    \
		if (hi > n) hi = n;                                                                    \
		job[t] = (bm_##SFX) { (const unsigned char *) pts, stride, lo, hi, nq, kinds, min1,    \
		                      max1, min2, cnt + (size_t) t * nq, pos + (size_t) t * nq,        \
		                      out_idx, 1 };                                                    \
	}                                                                                          \
	for (int pass = 1; pass <= (out_idx ? 2 : 1); pass++) {                                    \
		int started = 0;                                                                       \
		for (int t = 0; t < threads; t++) {                                                    \
			job[t].pass = pass;                                                                \
			if (pthread_create(&th[t], NULL, bm_run_##SFX, &job[t]) != 0)                      \
				break;                                                                         \
			started++;                                                                         \
		}                                                                                      \
		for (int t = 0; t < started; t++)                                                      \
			pthread_join(th[t], NULL);                                                         \
		if (started < threads)                                                                 \
			goto done;                                                                         \
		if (pass == 1) {                                                                       \
			/* query q's hits: thread 0's, then thread 1's, ... (index order) */              \
			uint64_t acc = 0;                                                                  \
			for (uint32_t q = 0; q < nq; q++) {                                                \
				out_off[q] = acc;                                                              \
				for (int t = 0; t < threads; t++) {                                            \
					pos[(size_t) t * nq + q] = acc;                                            \
					acc += cnt[(size_t) t * nq + q];                                           \
				}                                                                              \
			}                                                                                  \
			out_off[nq] = acc;                                                                 \
			total = (int64_t) acc;                                                             \
		}                                                                                      \
	}                                                                                          \
done:                                                                                          \
	free(job); free(th); free(cnt); free(pos);                                                 \
	return total;                                                                              \
}

BRUTE_MULTI_DEFINE(f32, float)
BRUTE_MULTI_DEFINE(f64, double)
BRUTE_MULTI_DEFINE(i32, int32_t)
