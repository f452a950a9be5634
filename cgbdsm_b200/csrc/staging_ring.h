// Staging ring of the serving loop: contiguous byte blocks allocated in FIFO
// order and released in the same order (a block is released when its batch
// completes; batches complete in submission order).  A block that would
// straddle the end of the ring starts at 0 instead, and the skipped end is
// accounted as used until the release that passes it.
#pragma once
#include <algorithm>
#include <cstdint>

namespace cgb {

struct StagingRing {
    uint64_t cap = 0;   // bytes
    uint64_t head = 0;  // first byte of the oldest live block
    uint64_t used = 0;  // bytes from head (live blocks and skipped ends)

    // Allocates len bytes (len > 0); false if they do not fit now.
    bool alloc(uint64_t len, uint64_t* off) {
        if (len == 0 || len > cap || used + len > cap) return false;
        uint64_t tail = (head + used) % cap;  // first free byte
        if (tail + len > cap) {               // wrap: skip the end of the ring
            const uint64_t skip = cap - tail;
            if (used + skip + len > cap) return false;
            used += skip;
            tail = 0;
        }
        *off = tail;
        used += len;
        return true;
    }

    // Releases the oldest live block [off, off + len), and any skipped end
    // before it.
    void release(uint64_t off, uint64_t len) {
        if (len == 0) return;
        const uint64_t end = off + len;
        const uint64_t freed = (end >= head) ? end - head : cap - head + end;
        used -= std::min(freed, used);
        head = end % cap;
        if (used == 0) head = 0;
    }
};

}  // namespace cgb
