// Test-only: stands where the reference's host-layer sources include "algorithms/plan.hpp"
// (src/plugin/roi.hpp:2, src/plugin/filter.hpp), so that those files compile against the
// B200 facade instead of the reference core. The reference's own base/checked.hpp provides
// the helpers they use (require, mul_size, checked_plane, checked_subplane).
#pragma once
#include "base/checked.hpp"
#include "neo_fft_b200/plan.hpp"
