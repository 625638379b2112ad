// pm_context.h -- the opaque handles behind the C ABI (include/polymult_b200.h).
#pragma once

#include "pm_batch.h"
#include "pm_engine.h"
#include "pm_server.h"

struct pm_context {
    pm::Engine* engine;
    double tuned_ms[2] = {0.0, 0.0};  // median pm_run of the schedule pm_tune_pipeline chose, per kind
};

struct pm_batch {
    pm::Batch* batch;
};

struct pm_server {
    pm::Server* server;
};
