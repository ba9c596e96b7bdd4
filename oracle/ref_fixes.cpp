// Test infrastructure: linked ahead of the reference library into
// oracle/_ref/kirchmig2d_cig_fwd only (the forward-modelling fixtures).
//
// The reference's adj=0 path reads the model with
// sep_read_fromsep(mig, nzx * ng, 0, &out[0], NULL) (src/kirchmig2d_cig.cpp:966)
// while sep_read_fromsep dereferences its size argument unconditionally
// (SEFILESYSTEM/src/se_fs_sep.cpp:1420-1430), so every adj=0 run stops with a
// null-pointer fault before modelling.  This helper does the same read and
// treats a missing size argument as "the buffer is large enough", which is
// what the call site means (out[0] holds nzx * ng floats).  Nothing else of
// the reference is replaced.
#include "se_fs_sep.h"

float *sep_read_fromsep(sep_t *sep, int64_t size, int64_t offset, float **buff, size_t *crt_size)
{
    if (crt_size && *crt_size < (size_t)size) {
        *crt_size = (size_t)size;
        *buff = realloc1float(*buff, *crt_size);
    }
    se_fsio_seek(sep->data->io, offset);
    se_fsio_read_float(sep->data->io, *buff, (size_t)size);
    return *buff;
}
