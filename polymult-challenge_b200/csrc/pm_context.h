// pm_context.h -- the opaque handle behind the C ABI (include/polymult_b200.h).
#pragma once

#include "pm_engine.h"

struct pm_context {
    pm::Engine* engine;
};
