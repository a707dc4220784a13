// Generated by gen_eri.py from data/class_table_b200.json.  Do not edit.
// Default MOLINTS_METHOD_AUTO table of contexts on the device named below:
// autotune.tune_class_methods on B200 (bench.py): 8 molecules of the 256-molecule batch and 4 serving requests, each class pair's HGP and Rys kernels (FP64 and MIXED) timed alone.
// Entries: 1 HGP, 2 Rys, | 4 (MOLINTS_CLASS_NO_FP32) where MIXED runs the FP64 kernel.
#pragma once
#include <stdint.h>
namespace molints {
constexpr const char *kTunedDevice = "NVIDIA B200";
static const int32_t kTunedClassMethods[11][11] = {
    {5, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {5, 5, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {5, 5, 5, 0, 0, 0, 0, 0, 0, 0, 0},
    {5, 5, 5, 5, 0, 0, 0, 0, 0, 0, 0},
    {5, 5, 5, 5, 6, 0, 0, 0, 0, 0, 0},
    {5, 5, 5, 5, 5, 5, 0, 0, 0, 0, 0},
    {5, 5, 5, 5, 5, 6, 6, 0, 0, 0, 0},
    {5, 5, 6, 5, 6, 6, 6, 6, 0, 0, 0},
    {6, 6, 6, 6, 2, 6, 6, 6, 6, 0, 0},
    {5, 5, 6, 6, 6, 6, 6, 6, 6, 6, 0},
    {5, 2, 6, 6, 6, 6, 6, 6, 6, 6, 6},
};
// work-queue schedule: lane_cost, hgp_widen, rys_chunks, rys_max_width, gather_blocks (autotune.tune_schedule on B200 (bench.py): a batch plan over 8 molecules of the 256-molecule batch, 54.8 ms with lane_cost 320 and 5 gather blocks per SM, 53.0 ms with this one)
static const double kTunedSchedule[5] = {640.0, 1.0, 4096.0, 8.0, 4.0};
}  // namespace molints
