/* gexs_tiles_gh32.cu — tile-kernel variants of profile class PK_GH32. */
#include "gexs_tiles.cuh"

namespace gexs {

cudaError_t launch_tiles_gh32(int prec, const KArgs& a, const gexs_launch_cfg& cfg, int nsm,
                              cudaStream_t st)
{
    return launch_pk<PK_GH32>(prec, a, cfg, nsm, st);
}

}  // namespace gexs
