// Admission rule of the serving loop (knng_server_*), host-only so that it can
// be tested without a device.  Jobs are admitted in arrival order: the job at
// the head of the queue starts once its HBM reservation fits next to the
// running jobs' reservations and a running slot is free; a later job never
// overtakes it.
#pragma once

#include <cstdint>

namespace knng {

// True when a job reserving `need` bytes may start now.
inline bool admits(uint64_t in_use, uint64_t need, uint64_t budget, uint32_t running, uint32_t max_running) {
    return running < max_running && in_use + need <= budget;
}

}  // namespace knng
