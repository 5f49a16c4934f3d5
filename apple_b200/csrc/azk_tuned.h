// Generated by `python -m apple_b200.autotune --export` from measured commit-kernel
// timings on sm100-148sm (4104 records) and the cost model trained on them;
// tests/test_tuned_tables.py keeps it equal to apple_b200/tuned_b200.json.
// Entry [k] = treelet depth (kTuned_*) and threads per CTA (kTunedThreads_*) for a layer
// of 2^k leaves (0: not used; the schedule's own value).
#pragma once
#include <stdint.h>

namespace azk {
static constexpr uint8_t kTuned_pcs_single[32] = {0, 1, 2, 3, 4, 5, 6, 7, 7, 8, 9, 7, 7, 8, 8, 8, 9, 10, 11, 12, 13, 12, 11, 11, 12, 12, 13, 0, 0, 0, 0, 0};
static constexpr uint8_t kTuned_pcs_batch[32] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 8, 9, 10, 11, 12, 13, 12, 13, 13, 11, 11, 12, 13, 13, 13, 13, 13, 13, 0, 0, 0, 0, 0};
static constexpr uint8_t kTuned_merkle_raw64[32] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 8, 7, 7, 8, 8, 7, 8, 9, 10, 11, 12, 10, 11, 12, 12, 12, 12, 13, 0, 0, 0, 0, 0};
static constexpr uint16_t kTunedThreads_pcs_single[32] = {0, 256, 512, 512, 512, 512, 512, 512, 256, 256, 256, 128, 128, 128, 128, 128, 512, 128, 256, 256, 256, 256, 128, 128, 128, 128, 128, 0, 0, 0, 0, 0};
static constexpr uint16_t kTunedThreads_pcs_batch[32] = {0, 256, 256, 256, 256, 256, 256, 256, 256, 256, 256, 256, 256, 256, 256, 256, 256, 256, 256, 256, 256, 256, 256, 256, 256, 256, 256, 0, 0, 0, 0, 0};
static constexpr uint16_t kTunedThreads_merkle_raw64[32] = {0, 256, 512, 512, 512, 128, 128, 256, 512, 128, 512, 512, 512, 512, 128, 128, 128, 128, 256, 512, 128, 128, 256, 256, 128, 128, 128, 0, 0, 0, 0, 0};
}  // namespace azk
