// Host-side FFT plan construction: factorisation of n into the radices the
// device butterflies implement, per-stage p values and twiddle / root tables
// computed in double precision and rounded once to float.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <map>
#include <string>
#include <vector>

#include "kernels.h"

namespace oks {

// Radices, largest power-of-two blocks first (16, 8, 4, 2), then 3, 5 and
// any remaining prime factor (handled by the generic direct-DFT butterfly).
inline std::vector<int> factorize(int n) {
    std::vector<int> r;
    int m = n;
    while (m % 16 == 0) { r.push_back(16); m /= 16; }
    if (m % 8 == 0) { r.push_back(8); m /= 8; }
    if (m % 4 == 0) { r.push_back(4); m /= 4; }
    if (m % 2 == 0) { r.push_back(2); m /= 2; }
    while (m % 3 == 0) { r.push_back(3); m /= 3; }
    while (m % 5 == 0) { r.push_back(5); m /= 5; }
    for (int f = 7; m > 1; f += 2) {
        while (m % f == 0) { r.push_back(f); m /= f; }
        if ((long long)f * f > m && m > 1) { r.push_back(m); m = 1; }
    }
    return r;
}

// Fills `pl` and the host tables for length n.  Returns false if n needs
// more stages than the plan holds.
inline bool build_plan(int n, FftPlan* pl, std::vector<float2>* tw, std::vector<float2>* roots) {
    std::vector<int> r = (n > 1) ? factorize(n) : std::vector<int>{};
    if ((int)r.size() > kMaxStages) return false;
    *pl = FftPlan{};
    pl->n = n;
    pl->nst = (int)r.size();
    tw->clear();
    roots->clear();
    const double two_pi = 6.283185307179586476925286766559;
    auto add_table = [&](int p, int R) {
        int off = (int)tw->size();
        for (int k = 0; k < p; ++k)
            for (int j = 1; j < R; ++j) {
                double a = -two_pi * (double)j * (double)k / ((double)p * R);
                tw->push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
            }
        return off;
    };
    int p = 1;
    for (int s = 0; s < pl->nst; ++s) {
        pl->rad[s] = r[s];
        pl->p_f[s] = p;
        pl->tw_f[s] = add_table(p, r[s]);
        p *= r[s];
    }
    p = 1;
    for (int s = 0; s < pl->nst; ++s) {
        const int R = r[pl->nst - 1 - s];
        pl->p_i[s] = p;
        pl->tw_i[s] = add_table(p, R);
        p *= R;
    }
    for (int s = 0; s < pl->nst; ++s) {
        pl->root_off[s] = (int)roots->size();
        for (int m = 0; m < r[s]; ++m) {
            double a = two_pi * (double)m / (double)r[s];
            roots->push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
        }
    }
    if (tw->empty()) tw->push_back(make_float2(1.f, 0.f));
    if (roots->empty()) roots->push_back(make_float2(1.f, 0.f));
    pl->tw_total = (int)tw->size();
    return true;
}

// Per-context cache of device plans keyed by length.
class PlanCache {
  public:
    ~PlanCache() { clear(); }
    const DevPlan* get(int n, std::string* err) {
        auto it = plans_.find(n);
        if (it != plans_.end()) return &it->second;
        DevPlan d;
        std::vector<float2> tw, roots;
        if (!build_plan(n, &d.plan, &tw, &roots)) {
            *err = "too many FFT stages";
            return nullptr;
        }
        cudaError_t e = cudaMalloc(&d.tw, sizeof(float2) * tw.size());
        if (e == cudaSuccess) e = cudaMalloc(&d.roots, sizeof(float2) * roots.size());
        if (e == cudaSuccess)
            e = cudaMemcpy(d.tw, tw.data(), sizeof(float2) * tw.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(d.roots, roots.data(), sizeof(float2) * roots.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            if (d.tw) cudaFree(d.tw);
            if (d.roots) cudaFree(d.roots);
            *err = cudaGetErrorString(e);
            return nullptr;
        }
        d.roots_total = (int)roots.size();
        return &(plans_[n] = d);
    }
    void clear() {
        for (auto& kv : plans_) {
            cudaFree(kv.second.tw);
            cudaFree(kv.second.roots);
        }
        plans_.clear();
    }

  private:
    std::map<int, DevPlan> plans_;
};

}  // namespace oks
