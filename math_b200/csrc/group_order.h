// Ordering of a pixel's sample group (src/painter/pixels/samples/com/sort.h),
// host and device.
#pragma once

#include "core.cuh"

namespace nbpt
{
inline constexpr int HELD_OUT = 4; // the reference's FILTER_SAMPLE_COUNT (pixels.h:42)

// ---------------------------------------------------------------------------
// ordering of a group: the steps of libstdc++'s insertion sort (for up to
// eight entries) and of its binary-heap partial selection (more entries), on
// an index array.

template <typename Less>
NBPT_HD void insertion_sort(int* a, const int n, const Less& less)
{
        for (int i = 1; i < n; ++i)
        {
                const int v = a[i];
                if (less(v, a[0]))
                {
                        for (int k = i; k > 0; --k)
                        {
                                a[k] = a[k - 1];
                        }
                        a[0] = v;
                }
                else
                {
                        int k = i;
                        while (less(v, a[k - 1]))
                        {
                                a[k] = a[k - 1];
                                --k;
                        }
                        a[k] = v;
                }
        }
}

// src/painter/pixels/samples/com/sort.h:26-46 on an index array ordered by
// key(index): up to 2 * HELD_OUT entries an insertion sort; more, the two
// smallest to the front and the two largest to the back by
// std::partial_sort (libstdc++ __heap_select + __sort_heap), once from each
// end.  With a heap of two entries those steps reduce to what follows: the
// heap is its top t and the other entry s; make_heap puts the larger of the
// first two on top; every later entry x that compares below the top takes
// the top's place in the array, and the new heap is {x on top, s} when s < x,
// else {s on top, x}; sort_heap leaves s, t.  The entries between keep the
// order these moves give them, the order the reference sums them in.
template <typename Key>
NBPT_HD void order_group(int* a, const int n, const Key& key)
{
        if (n <= 1)
        {
                return;
        }
        if (n <= HELD_OUT * 2)
        {
                insertion_sort(a, n, [&](const int x, const int y) { return key(x) < key(y); });
                return;
        }
        static_assert(HELD_OUT == 4);
        {
                // partial_sort(a, a + 2, a + n, less)
                int t = a[0];
                int s = a[1];
                float tk = key(t);
                float sk = key(s);
                if (!(sk < tk))
                {
                        const int i = t;
                        t = s;
                        s = i;
                        const float k = tk;
                        tk = sk;
                        sk = k;
                }
                for (int i = 2; i < n; ++i)
                {
                        const int x = a[i];
                        const float xk = key(x);
                        if (xk < tk)
                        {
                                a[i] = t;
                                if (sk < xk)
                                {
                                        t = x;
                                        tk = xk;
                                }
                                else
                                {
                                        t = s;
                                        tk = sk;
                                        s = x;
                                        sk = xk;
                                }
                        }
                }
                a[0] = s;
                a[1] = t;
        }
        {
                // partial_sort of [2, n) viewed from the end with greater: the
                // view's element j is a[n - 1 - j]
                int t = a[n - 1];
                int s = a[n - 2];
                float tk = key(t);
                float sk = key(s);
                if (!(sk > tk))
                {
                        const int i = t;
                        t = s;
                        s = i;
                        const float k = tk;
                        tk = sk;
                        sk = k;
                }
                for (int p = n - 3; p >= HELD_OUT / 2; --p)
                {
                        const int x = a[p];
                        const float xk = key(x);
                        if (xk > tk)
                        {
                                a[p] = t;
                                if (sk > xk)
                                {
                                        t = x;
                                        tk = xk;
                                }
                                else
                                {
                                        t = s;
                                        tk = sk;
                                        s = x;
                                        sk = xk;
                                }
                        }
                }
                a[n - 1] = s;
                a[n - 2] = t;
        }
}

} // namespace nbpt
