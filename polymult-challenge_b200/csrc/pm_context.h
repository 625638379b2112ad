// pm_context.h -- the opaque handles behind the C ABI (include/polymult_b200.h).
#pragma once

#include "pm_batch.h"
#include "pm_engine.h"
#include "pm_server.h"

struct pm_context {
    pm::Engine* engine;
};

struct pm_batch {
    pm::Batch* batch;
};

struct pm_server {
    pm::Server* server;
};
