// SPDX-License-Identifier: MIT
// Host-side tile planning for the listed-worlds tick (include/ebb.h: ebb_plan_worlds).
//
// Worlds are row runs anywhere in a park; a tile is any set of whole worlds of at most `cap` rows, so the planner is
// free to group worlds that are far apart. It packs them best-fit decreasing: the worlds by size, largest first, each
// into the open tile whose free rows fit it most tightly (or a new tile), which leaves few tiles and little idle room
// in each. Then every tile lists its worlds in row order, so that a tile's records pass reads memory in order.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "../../include/ebb.h"

extern "C" int64_t ebb_plan_worlds(const int64_t* starts, const int64_t* lens, int64_t count, int tile_cap,
                                   int64_t* worlds, int64_t* tile_worlds) {
    if (count < 0 || tile_cap <= 0 || tile_cap > EBB_WORLDS_MAX_TILE) return EBB_EINVAL;
    if (count == 0) {
        if (tile_worlds) tile_worlds[0] = 0;
        return 0;
    }
    if (!starts || !lens || !worlds || !tile_worlds) return EBB_EINVAL;
    // the worlds by size, largest first (a counting sort: sizes are at most tile_cap; equal sizes in input order)
    std::vector<int64_t> at((size_t)tile_cap + 2, 0);
    int64_t listed = 0;
    for (int64_t k = 0; k < count; ++k) {
        if (lens[k] > tile_cap || lens[k] < 0 || starts[k] < 0) return EBB_EINVAL;
        if (lens[k] > 0) {
            ++at[(size_t)(tile_cap - lens[k]) + 1];
            ++listed;
        }
    }
    for (int r = 0; r <= tile_cap; ++r) at[(size_t)r + 1] += at[(size_t)r];
    std::vector<int64_t> order((size_t)listed);
    for (int64_t k = 0; k < count; ++k)
        if (lens[k] > 0) order[(size_t)at[(size_t)(tile_cap - lens[k])]++] = k;
    // open tiles by free rows: bucket r holds the tiles with r rows free; `nonempty` marks the buckets in use
    const int words = tile_cap / 64 + 1;
    std::vector<std::vector<int32_t>> bucket((size_t)tile_cap + 1);
    std::vector<uint64_t> nonempty((size_t)words, 0);
    std::vector<int32_t> tile_of(order.size());
    int32_t tiles = 0;
    for (size_t q = 0; q < order.size(); ++q) {
        const int n = (int)lens[order[q]];
        int r = -1;                                                   // the least free-row count >= n in use
        for (int w = n / 64; w < words && r < 0; ++w) {
            uint64_t bits = nonempty[(size_t)w];
            if (w == n / 64) bits &= ~0ull << (n % 64);
            if (bits) r = w * 64 + __builtin_ctzll(bits);
        }
        int32_t t;
        if (r < 0) {
            t = tiles++;
            r = tile_cap;
        } else {
            t = bucket[(size_t)r].back();
            bucket[(size_t)r].pop_back();
            if (bucket[(size_t)r].empty()) nonempty[(size_t)(r / 64)] &= ~(1ull << (r % 64));
        }
        tile_of[q] = t;
        const int left = r - n;
        if (left > 0) {
            bucket[(size_t)left].push_back(t);
            nonempty[(size_t)(left / 64)] |= 1ull << (left % 64);
        }
    }
    // the worlds tile by tile, each tile's in row order
    std::vector<int64_t> first((size_t)tiles + 1, 0);
    for (size_t q = 0; q < order.size(); ++q) ++first[(size_t)tile_of[q] + 1];
    for (int32_t t = 0; t < tiles; ++t) first[(size_t)t + 1] += first[(size_t)t];
    std::vector<int64_t> fill(first.begin(), first.end() - 1);
    std::vector<int64_t> slot(order.size());
    for (size_t q = 0; q < order.size(); ++q) slot[(size_t)fill[(size_t)tile_of[q]]++] = order[q];
    for (int32_t t = 0; t < tiles; ++t)
        std::sort(slot.begin() + first[(size_t)t], slot.begin() + first[(size_t)t + 1],
                  [&](int64_t a, int64_t b) { return starts[a] < starts[b]; });
    for (size_t k = 0; k < slot.size(); ++k) {
        worlds[2 * k] = starts[slot[k]];
        worlds[2 * k + 1] = starts[slot[k]] + lens[slot[k]];
    }
    for (int32_t t = 0; t <= tiles; ++t) tile_worlds[t] = first[(size_t)t];
    return tiles;
}
