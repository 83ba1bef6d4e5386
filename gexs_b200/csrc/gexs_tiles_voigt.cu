/* gexs_tiles_voigt.cu — tile-kernel variants of profile class PK_VOIGT. */
#include "gexs_tiles.cuh"

namespace gexs {

cudaError_t launch_tiles_voigt(int prec, const KArgs& a, const gexs_launch_cfg& cfg, int nsm,
                               cudaStream_t st)
{
    return launch_pk<PK_VOIGT>(prec, a, cfg, nsm, st);
}

}  // namespace gexs
