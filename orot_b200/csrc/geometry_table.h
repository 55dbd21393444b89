// geometry_table.h -- pass geometry per pass-size class, read by Engine::plan.
//
// Written by `python -m orot_b200.tune` (the autotuner), which times every
// candidate on the device and keeps the fastest; this version holds the
// hand-set rules the tuner starts from.  A class applies to passes of at
// least min_bytes input bytes (on a 148-SM B200; other devices scale the
// bounds by their SM count).
//   tile12, tile14  fast-level tile bytes at 12 hash bits (level 1) and
//                   14 (levels 2-3): one warp walks one tile
//   lazy_run[g]     tiles per CTA run at levels 4-6, 7-9 and 10-12: one CTA
//                   slides its window over that many consecutive tiles
// Level 1-3 hash widths are fixed (parity with the reference); the output of
// a pass does not depend on any value here.
#pragma once
#include <cstdint>

namespace orotb {

struct GeometryRow {
  uint64_t min_bytes;
  uint32_t tile12, tile14;
  uint32_t lazy_run[3];
};

constexpr const char* kGeometrySource = "orot_b200.tune on NVIDIA B200, 148 SMs, 2026-12-04";
constexpr GeometryRow kGeometry[] = {
    {0ull, 4096, 8192, {1, 1, 1}},
    {1ull << 20, 4096, 8192, {2, 2, 2}},
    {4ull << 20, 4096, 8192, {8, 8, 1}},
    {16ull << 20, 16384, 16384, {4, 4, 4}},
    {64ull << 20, 16384, 16384, {16, 8, 4}},
    {256ull << 20, 32768, 32768, {16, 16, 16}},
    {1ull << 30, 32768, 65536, {32, 32, 16}},
    {4ull << 30, 65536, 65536, {32, 32, 16}},
};

}  // namespace orotb
