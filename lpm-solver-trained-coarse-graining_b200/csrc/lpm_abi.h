// Conversion of the C-ABI descriptors (lpm_lattice, lpm_batch, coefficient layout) to the library's internal structs,
// with the argument checks every entry point applies.  Shared by capi.cu and kmv_static.cu so that the entry points
// cannot drift apart.
#pragma once
#include <cstdint>

#include "../../include/lpm_b200.h"
#include "lpm_kernels.h"

namespace lpm {

// Validates a lattice descriptor and converts it.  Returns LPM_OK or LPM_ERR_ARG.
inline int to_lattice(const lpm_lattice* in, Lattice& L)
{
    if (!in) return LPM_ERR_ARG;
    if (in->dim != 2 && in->dim != 3) return LPM_ERR_ARG;
    if (in->nx < 1 || in->ny < 1 || in->nz < 1 || in->n < 1) return LPM_ERR_ARG;
    if (in->dim == 2 && in->nz != 1) return LPM_ERR_ARG;
    if (!in->nbr && in->n != (int64_t)in->nx * in->ny * in->nz) return LPM_ERR_ARG;
    if (in->n > INT64_C(1) << 40) return LPM_ERR_ARG;
    L.dim = in->dim;
    L.nx = in->nx;
    L.ny = in->ny;
    L.nz = in->nz;
    L.N = in->n;
    L.nbr = in->nbr;
    return LPM_OK;
}

inline int to_batch(const lpm_batch* in, Batch& b)
{
    if (!in || in->nsys < 1 || in->rhs_per_set < 1 || in->nmask < 1) return LPM_ERR_ARG;
    b.nsys = in->nsys;
    b.rhs_per_set = in->rhs_per_set;
    b.nmask = in->nmask;
    return LPM_OK;
}

inline int to_layout(int layout, const Lattice& L, CoefLayout& cl)
{
    const int NN = slots_of(L);
    cl.set_stride = L.N * NN;
    if (layout == LPM_LAYOUT_REF) {
        cl.slot_stride = 1;
        cl.site_stride = NN;
    } else if (layout == LPM_LAYOUT_SOA) {
        cl.slot_stride = L.N;
        cl.site_stride = 1;
    } else {
        return LPM_ERR_ARG;
    }
    return LPM_OK;
}

}  // namespace lpm
