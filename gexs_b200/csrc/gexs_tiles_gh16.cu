/* gexs_tiles_gh16.cu — tile-kernel variants of profile class PK_GH16. */
#include "gexs_tiles.cuh"

namespace gexs {

cudaError_t launch_tiles_gh16(int prec, const KArgs& a, const gexs_launch_cfg& cfg, int nsm,
                              cudaStream_t st)
{
    return launch_pk<PK_GH16>(prec, a, cfg, nsm, st);
}

}  // namespace gexs
