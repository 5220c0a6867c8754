// Low-octave desert proxy on zone grids (stage S4) -- see proxy kernels below.
#include "common.cuh"

namespace dsg {
namespace { float g_cut = 0.35f; }
void proxy_set_cut(float cut) { g_cut = cut; }
float proxy_cut() { return g_cut; }
}  // namespace dsg
