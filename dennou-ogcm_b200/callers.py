"""Batched forms of dogcm's per-level transform loops.

dogcm calls the SpmlUtil operators one level at a time inside `do k` loops
(dynamics/hspm_vfvm/HBEBaroc_hspm_vfvm_mod.f90:160-172 and :388-441,
dynamics/hspm_vfvm/HBEDiagnose_hspm_vfvm_mod.f90:276-284).  On the
GPU a per-level call is a handful of small kernel launches and is bound by
launch latency; the same loop as one call over all levels runs the kernels
once over K columns.  These functions are the spectral parts of those loops
written that way, on a SpmlUtil plan and CUDA float64 tensors of shape
(K, jm, im) (grids) or (K, lm) (spectra).  The grid-space terms the loops
build from the model state (the vertical flux divergence, the Coriolis and
pressure-gradient terms) are the caller's inputs.

`per_level` runs any of them level by level, the form the reference loops
have, for comparison and timing.
"""
from __future__ import annotations


def htrc_rhs(sp, u, v, tmp, vflx_div, adv_filter, h_phys):
    """Tracer tendency of HBEBaroc_HTRCRHS (HBEBaroc_hspm_vfvm_mod.f90:160-172):

        wz = -w_AlphaOptr_xy(U Tmp, V Tmp) + w_xy(vflx_div)
        xyz_HTRC_RHS = xy_w(w_AdvFilter wz) + h_phys

    with Tmp = H cos(phi) TRC and vflx_div = -(ADVFlxZ(k-1) - ADVFlxZ(k)) RCDK(k)
    given per level.  Three transform calls for all levels: the flux
    divergence with its products formed in the longitude transform, the
    analysis of the vertical term and the synthesis."""
    w = sp.w_xy(vflx_div) - sp.w_AlphaOptrProd_xy(u, v, tmp)
    w *= adv_filter[None, :]
    return sp.xy_w(w) + h_phys


def momrhs_vordiv(sp, a, b, c):
    """Velocity tendencies of HBEBaroc_MOMRHS_VorDivForm
    (HBEBaroc_hspm_vfvm_mod.f90:430-441), given the grid terms xy_A, xy_B
    (both already multiplied by cos(phi)) and xy_C of :396-428:

        w_Vor_RHS = -w_AlphaOptr_xy(A, B)
        w_Div_RHS =  w_AlphaOptr_xy(B, -A) - w_Lapla_w(w_xy(C))
        (U_RHS, V_RHS) = calc_VorDiv2UV(w_Vor_RHS, w_Div_RHS)

    calc_UVCosLat2VorDiv(A, B) returns (H(B, -A), H(A, B)) with H =
    w_AlphaOptr_xy, i.e. (w_Div_RHS + Lapla term, -w_Vor_RHS) from one
    analysis of both fields.  Four calls for all levels."""
    vor, div = sp.calc_UVCosLat2VorDiv(a, b)
    return sp.calc_VorDiv2UV(-div, vor - sp.w_Lapla_w(sp.w_xy(c)))


def momrhs_vordiv_fma(sp, u, v, vor, za, zb, c):
    """The same tendencies from the model's fields instead of xy_A, xy_B:

        xy_A = cos(phi) (Vor U + za),  xy_B = cos(phi) (Vor V + zb)

    (HBEBaroc_hspm_vfvm_mod.f90:394-418; za, zb every other term of the
    products, e.g. CoriU + VAdvV/H - VRHS_phys + DensEdd GradLat(GeoPot)/(rho a)),
    with the products formed while the grids load into the longitude
    transform, so that A and B are never written."""
    wv, wd = sp.calc_UVCosLat2VorDiv_fma(u, v, vor, za, zb)
    return sp.calc_VorDiv2UV(-wd, wv - sp.w_Lapla_w(sp.w_xy(c)))


def diagnose_vordiv(sp, u, v):
    """Vorticity and divergence grids of HBEDiagnose_VorDiv
    (HBEDiagnose_hspm_vfvm_mod.f90:276-284):

        (w_Vor, w_Div) = calc_UVCosLat2VorDiv(U cos(phi), V cos(phi))
        xyz_Vor = xy_w(w_Vor), xyz_Div = xy_w(w_Div)

    One analysis of both fields and one synthesis of 2 K columns."""
    import torch

    cs = torch.cos(torch.as_tensor(sp.y_Lat, dtype=torch.float64, device=u.device))[None, :, None]
    vor, div = sp.calc_UVCosLat2VorDiv(u * cs, v * cs)
    K = u.shape[0]
    g = sp.xy_w(torch.cat([vor, div]))
    return g[:K], g[K:]


def per_level(fn, sp, *arrays, **kw):
    """Run fn level by level (arrays with a leading level axis are sliced,
    others passed whole) and stack the results, as the reference's `do k`
    loops do."""
    import torch

    K = arrays[0].shape[0]
    outs = []
    for k in range(K):
        args = [x[k:k + 1] if (hasattr(x, "shape") and x.dim() >= 2 and x.shape[0] == K) else x for x in arrays]
        outs.append(fn(sp, *args, **kw))
    if isinstance(outs[0], tuple):
        return tuple(torch.cat([o[i] for o in outs]) for i in range(len(outs[0])))
    return torch.cat(outs)
