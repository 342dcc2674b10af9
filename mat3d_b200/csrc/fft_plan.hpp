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
// barrier fewer -- for callers whose kernels compile the 9-point butterfly)
inline bool make_plan(int n, LinePlan& p, bool fuse9 = false) {
    std::vector<int> f, odd;
    int m = n;
    int p2 = 0;
    while (m % 2 == 0) { ++p2; m /= 2; }
    if (fuse9)
        while (m % 9 == 0) { odd.push_back(9); m /= 9; }
    for (int q = 3; q <= m; q += 2)
        while (m % q == 0) { odd.push_back(q); m /= q; }
    std::sort(odd.begin(), odd.end());
    for (auto it = odd.rbegin(); it != odd.rend(); ++it) f.push_back(*it);
    for (; p2 >= 3; p2 -= 3) f.push_back(8);
    if (p2 == 2) f.push_back(4);
    if (p2 == 1) f.push_back(2);
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
