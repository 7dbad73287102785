// Tie-exact restatement of the sorting algorithm the reference relies on.
//
// The reference orders neighbour candidates with std::sort on entries compared
// by covariance only (sugarbox_indexed_neighbour_lookup.h:14-21,100) and
// orders its search template the same way (covariance_field.h:359). std::sort
// is not stable, so when several candidates share a covariance value the
// reference's choice among them is whatever permutation GNU libstdc++ (GCC 13,
// the toolchain the reference is built with here) produces. To pick the same
// members of a tie group that straddles the k-th slot, the device re-runs that
// algorithm on the candidate list. This file states the published algorithm of
// libstdc++'s std::sort in this project's own iterative form:
//
//   1. introsort loop: while a range holds more than 16 elements, either (if its
//      depth budget, initially 2*floor(log2 n), is spent) heap-sort it, or move
//      the median of {second, middle, last} elements to the front, partition the
//      rest around it with an unguarded Hoare scan (both scans stop on equal
//      keys), and continue on both sides with the budget decremented once;
//   2. heap sort: bottom-up make-heap with hole sifting (descend to a leaf via the
//      larger child, preferring the right one unless it is smaller than the left,
//      then bubble the value back up), then repeated pop-to-the-end;
//   3. final insertion sort over the whole array: guarded for the first 16
//      elements, unguarded for the rest.
//
// Sub-ranges produced by a partition are disjoint and each is processed from
// its own contents and depth budget only, so the order in which the explicit
// stack below visits them does not change the resulting permutation.
//
// Elements are compared with `less(a, b)`; every comparison and move of the
// published algorithm happens here in the same order, so any key type with a
// strict weak order gives the identical permutation.
#pragma once

#ifdef __CUDACC__
#define GIS_HD __host__ __device__ __forceinline__
#else
#define GIS_HD inline
#endif

namespace gis
{
template <typename E>
GIS_HD void swap_elems(E *a, long i, long j)
{
    E t = a[i];
    a[i] = a[j];
    a[j] = t;
}

// Places the median of a[x], a[y], a[z] at a[dst] by one swap.
template <typename E, typename Less>
GIS_HD void median_to_front(E *a, long dst, long x, long y, long z, Less less)
{
    long pick;
    if (less(a[x], a[y]))
        pick = less(a[y], a[z]) ? y : (less(a[x], a[z]) ? z : x);
    else
        pick = less(a[x], a[z]) ? x : (less(a[y], a[z]) ? z : y);
    swap_elems(a, dst, pick);
}

// Unguarded partition of (lo, hi) around the pivot held at a[lo].
template <typename E, typename Less>
GIS_HD long partition_around_front(E *a, long lo, long hi, Less less)
{
    long i = lo + 1, j = hi;
    for (;;)
    {
        while (less(a[i], a[lo])) ++i;
        --j;
        while (less(a[lo], a[j])) --j;
        if (!(i < j)) return i;
        swap_elems(a, i, j);
        ++i;
    }
}

// Hole sift within the heap a[base .. base+len): the hole at `hole` descends to
// a leaf, then `v` rises from there but not above `top`.
template <typename E, typename Less>
GIS_HD void heap_sift(E *a, long base, long hole, long len, E v, Less less)
{
    const long top = hole;
    long child = hole;
    while (child < (len - 1) / 2)
    {
        child = 2 * (child + 1);
        if (less(a[base + child], a[base + child - 1])) --child;
        a[base + hole] = a[base + child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2)
    {
        child = 2 * (child + 1);
        a[base + hole] = a[base + child - 1];
        hole = child - 1;
    }
    long parent = (hole - 1) / 2;
    while (hole > top && less(a[base + parent], v))
    {
        a[base + hole] = a[base + parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    a[base + hole] = v;
}

template <typename E, typename Less>
GIS_HD void heap_sort_range(E *a, long lo, long hi, Less less)
{
    const long len = hi - lo;
    if (len >= 2)
    {
        for (long p = (len - 2) / 2;; --p)
        {
            heap_sift(a, lo, p, len, a[lo + p], less);
            if (p == 0) break;
        }
    }
    for (long end = hi; end - lo > 1;)
    {
        --end;
        E v = a[end];
        a[end] = a[lo];
        heap_sift(a, lo, 0, end - lo, v, less);
    }
}

// Shifts a[i] left while it is less than its predecessor (no lower bound check:
// the caller guarantees an element not greater than it sits to the left).
template <typename E, typename Less>
GIS_HD void insert_unguarded(E *a, long i, Less less)
{
    E v = a[i];
    long k = i;
    while (less(v, a[k - 1]))
    {
        a[k] = a[k - 1];
        --k;
    }
    a[k] = v;
}

template <typename E, typename Less>
GIS_HD void insertion_sort_guarded(E *a, long lo, long hi, Less less)
{
    if (lo == hi) return;
    for (long i = lo + 1; i < hi; ++i)
    {
        if (less(a[i], a[lo]))
        {
            E v = a[i];
            for (long k = i; k > lo; --k) a[k] = a[k - 1];
            a[lo] = v;
        }
        else
        {
            insert_unguarded(a, i, less);
        }
    }
}

GIS_HD int floor_log2(long n)
{
    int r = 0;
    while (n > 1)
    {
        n >>= 1;
        ++r;
    }
    return r;
}

// Sorts a[0 .. n) and reproduces std::sort's permutation (see the file comment).
template <typename E, typename Less>
GIS_HD void sort(E *a, long n, Less less)
{
    const long kThreshold = 16;
    if (n <= 0) return;
    // explicit stack of pending (lo, hi, depth) ranges; at most one pending
    // range per depth level, and the budget is below 64 for any n < 2^31
    long st_lo[64], st_hi[64];
    int st_d[64];
    int sp = 0;
    st_lo[0] = 0;
    st_hi[0] = n;
    st_d[0] = 2 * floor_log2(n);
    sp = 1;
    while (sp > 0)
    {
        --sp;
        long lo = st_lo[sp], hi = st_hi[sp];
        int depth = st_d[sp];
        while (hi - lo > kThreshold)
        {
            if (depth == 0)
            {
                heap_sort_range(a, lo, hi, less);
                break;
            }
            --depth;
            long mid = lo + (hi - lo) / 2;
            median_to_front(a, lo, lo + 1, mid, hi - 1, less);
            long cut = partition_around_front(a, lo, hi, less);
            st_lo[sp] = cut;
            st_hi[sp] = hi;
            st_d[sp] = depth;
            ++sp;
            hi = cut;
        }
    }
    if (n > kThreshold)
    {
        insertion_sort_guarded(a, 0, kThreshold, less);
        for (long i = kThreshold; i < n; ++i) insert_unguarded(a, i, less);
    }
    else
    {
        insertion_sort_guarded(a, 0, n, less);
    }
}
// Rearranges a[0 .. n) so that a[0 .. k) holds exactly the elements that
// sort() (std::sort) places at positions 0 .. k-1; they are not put in order.
// Only the partitions of the ranges containing the boundary between positions
// k-1 and k are replayed: a partition leaves every element left of its cut not
// greater than every element right of it, later steps on a range only permute
// inside it, and the closing insertion sort is stable and never moves an
// element out of its final chunk of <= 16, so the chunk straddling the
// boundary is the only one whose internal order decides the split.
template <typename E, typename Less>
GIS_HD void select_first_k(E *a, long n, long k, Less less)
{
    const long kThreshold = 16;
    if (n <= 0 || k <= 0 || k >= n) return;
    long lo = 0, hi = n;
    int depth = 2 * floor_log2(n);
    while (hi - lo > kThreshold)
    {
        if (depth == 0)
        {
            heap_sort_range(a, lo, hi, less);
            return;
        }
        --depth;
        long mid = lo + (hi - lo) / 2;
        median_to_front(a, lo, lo + 1, mid, hi - 1, less);
        long cut = partition_around_front(a, lo, hi, less);
        if (cut == k) return;
        if (cut > k)
            hi = cut;
        else
            lo = cut;
    }
    insertion_sort_guarded(a, lo, hi, less);
}
} // namespace gis
