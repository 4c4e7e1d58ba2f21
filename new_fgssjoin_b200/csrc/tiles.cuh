// tiles.cuh -- the tile table of a batch of joins: per-record kernels cover
// every join of a batch in tiles of `tile` records of one join (no tile spans
// two joins, so a block's reductions belong to one join).  Join j's records
// are the batch's records [roff[j], roff[j+1]); tile_off[j] is its first tile.
#pragma once

#include <stdint.h>

namespace fgss {

struct TileMap {
    const uint32_t* tile_off;  // [nj + 1] first tile of each join
    const uint64_t* roff;      // [nj + 1] first record of each join in the batch's record space
    uint32_t nj;
    uint32_t tile;             // records per tile
    uint32_t ntiles;
};

// The join of tile b: the last j with tile_off[j] <= b.
__device__ __forceinline__ uint32_t tile_join(const TileMap& m, uint32_t b) {
    uint32_t lo = 0, hi = m.nj;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(m.tile_off + mid + 1) <= b) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Tile b's join j and its records [r0, r1) within the join.
struct TileRange {
    uint32_t j, r0, r1;
};
__device__ __forceinline__ TileRange tile_range(const TileMap& m, uint32_t b) {
    TileRange t;
    t.j = tile_join(m, b);
    t.r0 = (b - __ldg(m.tile_off + t.j)) * m.tile;
    const uint64_t n = __ldg(m.roff + t.j + 1) - __ldg(m.roff + t.j);
    t.r1 = (uint32_t)min((uint64_t)t.r0 + m.tile, n);
    return t;
}

}  // namespace fgss
