// Process-wide cache of cuFFT plans for the line-of-sight and correlation-function entries.
//
// Making a plan costs host time on every call of an entry (and the workspace queries make one
// only to learn its work-area size), so plans are kept, keyed on the device they were made on,
// the transform type and the batch shape.  Every plan is made with auto-allocation off: each call
// passes its own work area (a slice of the caller's workspace) and stream before executing, under
// the cache's mutex, so calls from several host threads or streams never share a work area.  The
// cache holds at most kFftPlanCacheSize plans; the oldest is destroyed to make room.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>

#include <mutex>
#include <vector>

namespace discoeb_fft {

constexpr size_t kFftPlanCacheSize = 16;

struct PlanKey {
    int dev;
    int type;  // cufftType
    long long n, batch, in_pitch, out_pitch;
    bool operator==(const PlanKey& o) const
    {
        return dev == o.dev && type == o.type && n == o.n && batch == o.batch && in_pitch == o.in_pitch &&
               out_pitch == o.out_pitch;
    }
};

struct PlanEntry {
    PlanKey key;
    cufftHandle plan;
    size_t work;
};

inline std::mutex& plan_mutex()
{
    static std::mutex mu;
    return mu;
}

inline std::vector<PlanEntry>& plan_entries()
{
    static std::vector<PlanEntry> entries;
    return entries;
}

// The plan of a batch of 1-D transforms of length n (rows `in_pitch` / `out_pitch` elements apart
// in the input / output) on the current device, made on first use.  The caller holds
// plan_mutex() from this call until its execution has been enqueued.  Returns false when cuFFT
// cannot make the plan.
inline bool cached_plan(cufftType type, long long n, long long batch, long long in_pitch, long long out_pitch,
                        cufftHandle* plan, size_t* work)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    const PlanKey key{dev, (int)type, n, batch, in_pitch, out_pitch};
    std::vector<PlanEntry>& entries = plan_entries();
    for (const PlanEntry& e : entries)
        if (e.key == key) {
            *plan = e.plan;
            *work = e.work;
            return true;
        }
    cufftHandle h;
    if (cufftCreate(&h) != CUFFT_SUCCESS) return false;
    cufftSetAutoAllocation(h, 0);
    long long nn[1] = {n}, inembed[1] = {in_pitch}, onembed[1] = {out_pitch};
    size_t ws = 0;
    if (cufftMakePlanMany64(h, 1, nn, inembed, 1, in_pitch, onembed, 1, out_pitch, type, batch, &ws) !=
        CUFFT_SUCCESS) {
        cufftDestroy(h);
        return false;
    }
    if (entries.size() >= kFftPlanCacheSize) {
        cufftDestroy(entries.front().plan);
        entries.erase(entries.begin());
    }
    entries.push_back({key, h, ws});
    *plan = h;
    *work = ws;
    return true;
}

}  // namespace discoeb_fft
