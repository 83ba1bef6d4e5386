/* gexs_tiles_erf.cu — tile-kernel variants of profile class PK_ERF. */
#include "gexs_tiles.cuh"

namespace gexs {

cudaError_t launch_tiles_erf(int prec, const KArgs& a, const gexs_launch_cfg& cfg, int nsm,
                             cudaStream_t st)
{
    return launch_pk<PK_ERF>(prec, a, cfg, nsm, st);
}

}  // namespace gexs
