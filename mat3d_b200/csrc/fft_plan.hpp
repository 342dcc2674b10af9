// fft_plan.hpp -- host-side set-up of the generic line FFTs: the radix
// schedule of a length and its twiddle table (shared by the 3-D and 2-D solvers).
#pragma once
#include <algorithm>
#include <cmath>
#include <vector>

#include "fft_smem.cuh"

namespace m3d {

// radix schedule: odd primes up to kMaxGenericRadix, largest first (the
// first stage needs no twiddle multiplications, so the costliest butterfly
// goes there), then 8, 4, 2; false if a factor is larger
// (fuse9: two factors 3 become one radix-9 stage -- one Stockham stage and
// barrier fewer -- for callers whose kernels compile the 9-point butterfly).
// Any order of the factors is a valid Stockham schedule; `order` picks one
// for the autotuner: 0 the above, 1 odd factors smallest first, 2 the
// power-of-two stages first, 3 the power of two as radix-4 stages (and one 2).
constexpr int kPlanOrders = 4;
inline bool make_plan(int n, LinePlan& p, bool fuse9 = false, int order = 0) {
    std::vector<int> f, odd;
    int m = n;
    int p2 = 0;
    while (m % 2 == 0) { ++p2; m /= 2; }
    if (fuse9)
        while (m % 9 == 0) { odd.push_back(9); m /= 9; }
    for (int q = 3; q <= m; q += 2)
        while (m % q == 0) { odd.push_back(q); m /= q; }
    std::sort(odd.begin(), odd.end());
    std::vector<int> pow2;
    if (order == 3) {
        for (; p2 >= 2; p2 -= 2) pow2.push_back(4);
    } else {
        for (; p2 >= 3; p2 -= 3) pow2.push_back(8);
        if (p2 == 2) pow2.push_back(4);
    }
    if (p2 == 1) pow2.push_back(2);
    if (order == 2) f = pow2;
    if (order == 1) f.insert(f.end(), odd.begin(), odd.end());
    else f.insert(f.end(), odd.rbegin(), odd.rend());
    if (order != 2) f.insert(f.end(), pow2.begin(), pow2.end());
    if (f.empty()) f.push_back(1);
    if ((int)f.size() > kMaxStages) return false;
    for (int r : f)
        if (r > kMaxGenericRadix) return false;
    p.n = n;
    p.nstages = (n == 1) ? 0 : (int)f.size();
    for (int i = 0; i < kMaxStages; ++i) p.radix[i] = i < (int)f.size() ? f[i] : 1;
    return true;
}

// tw[m] = exp(-2 pi i m / n), evaluated in long double
template <typename T>
inline std::vector<typename Cx<T>::t> twiddles(int n) {
    std::vector<typename Cx<T>::t> t(n);
    const long double two_pi = 6.283185307179586476925286766559L;
    for (int m = 0; m < n; ++m) {
        const long double a = -two_pi * (long double)m / (long double)n;
        t[m].x = (T)cosl(a);
        t[m].y = (T)sinl(a);
    }
    return t;
}

}  // namespace m3d
