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

// Radices: largest power-of-two blocks first (16, 8, 4, 2), then 3, 5 and
// any remaining prime factor (handled by the generic direct-DFT butterfly).
// Fills `pl` and writes the twiddle / root tables for length n into the
// caller's arrays (capacities tw_cap, roots_cap entries; no allocation).
// Returns false if n needs more stages than the plan holds or a table does
// not fit.  *tw_n / *roots_n receive the entry counts (at least 1 each).
inline bool build_plan_into(int n, FftPlan* pl, float2* tw, int tw_cap, int* tw_n, float2* roots, int roots_cap,
                            int* roots_n) {
    int r[64];
    int nr = 0;
    {
        int m = n > 1 ? n : 1;
        while (m % 16 == 0 && nr < 64) { r[nr++] = 16; m /= 16; }
        if (m % 8 == 0) { r[nr++] = 8; m /= 8; }
        if (m % 4 == 0) { r[nr++] = 4; m /= 4; }
        if (m % 2 == 0) { r[nr++] = 2; m /= 2; }
        while (m % 3 == 0 && nr < 64) { r[nr++] = 3; m /= 3; }
        while (m % 5 == 0 && nr < 64) { r[nr++] = 5; m /= 5; }
        for (int f = 7; m > 1 && nr < 64; f += 2) {
            while (m % f == 0 && nr < 64) { r[nr++] = f; m /= f; }
            if ((long long)f * f > m && m > 1) { r[nr++] = m; m = 1; }
        }
    }
    if (nr > kMaxStages) return false;
    *pl = FftPlan{};
    pl->n = n;
    pl->nst = nr;
    int nt = 0, nro = 0;
    const double two_pi = 6.283185307179586476925286766559;
    auto add_table = [&](int p, int R) -> int {
        const int off = nt;
        if ((long long)nt + (long long)p * (R - 1) > tw_cap) return -1;
        for (int k = 0; k < p; ++k)
            for (int j = 1; j < R; ++j) {
                double a = -two_pi * (double)j * (double)k / ((double)p * R);
                tw[nt++] = make_float2((float)std::cos(a), (float)std::sin(a));
            }
        return off;
    };
    int p = 1;
    for (int s = 0; s < nr; ++s) {
        pl->rad[s] = r[s];
        pl->p_f[s] = p;
        if ((pl->tw_f[s] = add_table(p, r[s])) < 0) return false;
        p *= r[s];
    }
    p = 1;
    for (int s = 0; s < nr; ++s) {
        const int R = r[nr - 1 - s];
        pl->p_i[s] = p;
        if ((pl->tw_i[s] = add_table(p, R)) < 0) return false;
        p *= R;
    }
    for (int s = 0; s < nr; ++s) {
        pl->root_off[s] = nro;
        if (nro + r[s] > roots_cap) return false;
        for (int m = 0; m < r[s]; ++m) {
            double a = two_pi * (double)m / (double)r[s];
            roots[nro++] = make_float2((float)std::cos(a), (float)std::sin(a));
        }
    }
    if (nt == 0) {
        if (tw_cap < 1) return false;
        tw[nt++] = make_float2(1.f, 0.f);
    }
    if (nro == 0) {
        if (roots_cap < 1) return false;
        roots[nro++] = make_float2(1.f, 0.f);
    }
    pl->tw_total = nt;
    *tw_n = nt;
    *roots_n = nro;
    return true;
}

// Vector form of build_plan_into.
inline bool build_plan(int n, FftPlan* pl, std::vector<float2>* tw, std::vector<float2>* roots) {
    // forward + inverse tables hold fewer than 2n entries; roots fewer than n + 1
    const int cap_tw = 2 * (n > 1 ? n : 1) + 1, cap_rt = (n > 1 ? n : 1) + 1;
    tw->assign(cap_tw, make_float2(0.f, 0.f));
    roots->assign(cap_rt, make_float2(0.f, 0.f));
    int ntw = 0, nrt = 0;
    if (!build_plan_into(n, pl, tw->data(), cap_tw, &ntw, roots->data(), cap_rt, &nrt)) return false;
    tw->resize(ntw);
    roots->resize(nrt);
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
