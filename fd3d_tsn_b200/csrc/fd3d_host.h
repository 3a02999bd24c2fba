// fd3d_host.h -- host-side helpers of the C ABI: result files and input decks.
#pragma once
#include "../../include/fd3d_gpu.h"

namespace fd3d {
// Appends every history record produced since `rec_written` to the reference's
// stream files under dir (sliprateX/Z.res, shearstressX/Z.res, psi.res for FVW,
// stan<i>.txt), and, once the solve has reached ntfd steps, writes the post-loop
// planes (ruptime.res, risetime.res, slipX/Z.res, stressdropX/Z.res, contour.res,
// czone.res, rvel.res).
int write_results(fd3d_ctx* ctx, const fd3d_params& p, int nf, int& rec_written, const char* dir, int real_kind);
}
