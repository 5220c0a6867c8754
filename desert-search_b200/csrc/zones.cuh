// Zone grids of the low-octave proxy (stage S4) as the device sees them, shared by the proxy kernels and the
// device-resident searcher that builds zones on the device.
#pragma once
#include <cstdint>
#include "kernels_tuned.h"

namespace dsg {
namespace zones {
// One zone: origin in quarts, step-32 cells nx x nz (row-major, z outer), its first cell in the concatenated
// bitmap, and the index of its seed's noise tables.
struct DZone { int32_t x0, z0, nx, nz; int64_t off; int32_t seed, pad; };
constexpr int CHUNK = DSG_ZONE_CHUNK;       // cells per block step of the zone kernels
// Chunk list of zones built on the device: chunk k covers cells [chunk[k].y * CHUNK, + CHUNK) of zone chunk[k].x.
// A null chunk list means the host-known layout: zone blockIdx.x, chunk blockIdx.y.
struct ZoneWork { const uint2 *chunk; const uint32_t *nchunk; };
// Statistics of one 8-connected component of a zone bitmap.  sx, sz: sums of the cells' columns and rows
// (exact integers); kid: index among the kept components or -1; seg, cur: its interior-key segment.
struct CompStat { uint32_t zone, first, cells, inner; int32_t minx, minz, kid; uint32_t seg, cur, pad; uint64_t sx, sz; };
}  // namespace zones
}  // namespace dsg
