// Hydrodynamic interaction: NEI_LIST_PRECOMP (partlib.f90:3218-3371), AFUN_PRECOMP
// (3375-3510) and HDI_GMRES (2795-3005).
#include "dl_internal.cuh"

int launch_nei_list(dl_ctx *c)
{
    return dl_fail(c, DL_E_STATE, "NEI_LIST_PRECOMP: not available in this build");
}

int run_gmres(dl_ctx *c, dl_gmres_report *)
{
    return dl_fail(c, DL_E_STATE, "HDI_GMRES: not available in this build");
}

extern "C" int dl_nei_list_precomp(dl_ctx *c)
{
    if (!c) return DL_E_ARG;
    return launch_nei_list(c);
}

extern "C" int dl_hdi_gmres(dl_ctx *c, dl_gmres_report *rep)
{
    if (!c) return DL_E_ARG;
    return run_gmres(c, rep);
}

extern "C" int dl_get_nei(dl_ctx *c, int *, int *, double *, int, int *nnz)
{
    if (!c) return DL_E_ARG;
    if (nnz) *nnz = 0;
    return dl_fail(c, DL_E_STATE, "dl_get_nei: not available in this build");
}
