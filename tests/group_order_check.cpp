// Checks order_group (math_b200/csrc/group_order.h) against libstdc++'s own
// std::sort and std::partial_sort as the reference's group sort calls them
// (src/painter/pixels/samples/com/sort.h:26-46), on seeded random groups with
// many equal keys.  Prints the number of mismatching groups.
#include "../math_b200/csrc/group_order.h"

#include <algorithm>
#include <cstdio>
#include <random>
#include <vector>

int main()
{
        std::mt19937 engine(12345);
        long mismatches = 0;
        long groups = 0;
        for (int n = 0; n <= 300; ++n)
        {
                for (int rep = 0; rep < 60; ++rep)
                {
                        // few distinct keys in half of the cases: ties everywhere
                        const int distinct = (rep % 2 == 0) ? 1 + static_cast<int>(engine() % 4) : 1000000;
                        std::vector<float> key(n);
                        for (float& k : key)
                        {
                                k = static_cast<float>(engine() % distinct) * 0.25f;
                        }
                        std::vector<int> ref(n);
                        for (int i = 0; i < n; ++i)
                        {
                                ref[i] = i;
                        }
                        std::vector<int> mine = ref;
                        const auto less = [&](const int a, const int b) { return key[a] < key[b]; };
                        const auto greater = [&](const int a, const int b) { return key[a] > key[b]; };
                        if (n > 1)
                        {
                                if (n <= 2 * nbpt::HELD_OUT)
                                {
                                        std::sort(ref.begin(), ref.end(), less);
                                }
                                else
                                {
                                        std::partial_sort(ref.begin(), ref.begin() + nbpt::HELD_OUT / 2, ref.end(), less);
                                        std::partial_sort(ref.rbegin(), ref.rbegin() + nbpt::HELD_OUT / 2,
                                                          ref.rend() - nbpt::HELD_OUT / 2, greater);
                                }
                        }
                        nbpt::order_group(mine.data(), n, [&](const int i) { return key[i]; });
                        ++groups;
                        mismatches += (mine != ref) ? 1 : 0;
                }
        }
        std::printf("%ld %ld\n", groups, mismatches);
        return 0;
}
