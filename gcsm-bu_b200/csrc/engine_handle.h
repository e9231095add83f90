// The opaque csm_engine handle of the C ABI: one Engine per handle.
#pragma once

#include "engine.h"

struct csm_engine {
    csm::Engine impl;
    explicit csm_engine(const csm_config &c) : impl(c) {}
};
