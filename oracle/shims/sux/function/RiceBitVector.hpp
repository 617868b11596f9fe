// Test infrastructure only (the oracle). The reference includes sux's RiceBitVector but uses its
// own fork (include/shockhash/RiceBitVector.h); nothing from this header is needed.
#pragma once
#include <sux/util/Vector.hpp>
#include <sux/support/common.hpp>
