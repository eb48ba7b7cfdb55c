"""The CPML-first tile order (IFOS_OPT_TILE_ORDER 2 and 3) as a map of the
spatial rank to a tile: the same closed form as cpml_first() in
ifos_b200/csrc/ifos_tile.cuh, checked here to be a permutation of the tiles
that ranks every tile meeting a CPML strip (the tiles the ops take their
slower CPML path on) before every interior tile, over grids whose strips
span fractions of tiles, whole tiles, overlap, or are absent.  The device
form is checked on the GPU by running every order bit-identical to the
others (tests/test_graphs_options.py)."""
import pytest

TX = 64


def cpml_first(rank, ntx, nty, ty_h, nx, ny, fw, free_surf):
    if fw <= 0:
        return rank
    cl = min(ntx, (fw - 1) // TX + 1)
    vx = nx - fw + 1 - TX
    xr0 = max(cl, 0 if vx <= 0 else (vx + TX - 1) // TX)
    rt = 0 if free_surf else min(nty, (fw - 1) // ty_h + 1)
    vy = ny - fw + 1 - ty_h
    yb0 = min(nty, max(rt, 0 if vy <= 0 else (vy + ty_h - 1) // ty_h))
    nys = rt + (nty - yb0)
    if rank < nys * ntx:
        r = rank // ntx
        return (r if r < rt else yb0 + (r - rt)) * ntx + (rank - r * ntx)
    rank -= nys * ntx
    ce = cl + (ntx - xr0)
    mid = nty - nys
    if rank < mid * ce:
        r, c = divmod(rank, ce)
        return (rt + r) * ntx + (c if c < cl else xr0 + (c - cl))
    rank -= mid * ce
    w = ntx - ce
    r, c = divmod(rank, w)
    return (rt + r) * ntx + cl + c


def in_strip(idx, ntx, ty_h, nx, ny, fw, free_surf):
    ty, tx = divmod(idx, ntx)
    i0, j0 = tx * TX + 1, ty * ty_h + 1
    i1 = min(i0 + TX - 1, nx)
    x = fw > 0 and (i0 <= fw or i1 >= nx - fw + 1)
    y = fw > 0 and ((not free_surf and j0 <= fw) or j0 + ty_h - 1 >= ny - fw + 1)
    return x or y


@pytest.mark.parametrize("nx,ny,fw,free_surf,ty_h", [
    (2000, 600, 30, 1, 8), (2000, 600, 30, 0, 8), (400, 160, 10, 1, 8), (4000, 1200, 40, 1, 8),
    (131, 37, 10, 1, 8), (64, 8, 3, 0, 8), (130, 40, 64, 0, 8), (130, 40, 65, 1, 8), (200, 50, 0, 1, 8),
    (77, 29, 6, 0, 16), (1000, 300, 100, 0, 8), (65, 17, 32, 0, 8)])
def test_cpml_first_is_a_permutation_with_strips_first(nx, ny, fw, free_surf, ty_h):
    ntx, nty = (nx + TX - 1) // TX, (ny + ty_h - 1) // ty_h
    n = ntx * nty
    seq = [cpml_first(r, ntx, nty, ty_h, nx, ny, fw, free_surf) for r in range(n)]
    assert sorted(seq) == list(range(n))
    flags = [in_strip(i, ntx, ty_h, nx, ny, fw, free_surf) for i in seq]
    k = sum(flags)
    assert all(flags[:k]) and not any(flags[k:])


def test_strip_tiles_spread_over_the_ctas():
    """Round-robin over 444 CTAs: the 2000 x 600 grid's strip tiles fall one
    per CTA at most, per shot, where the row-major order gives some CTAs
    none and others several."""
    nx, ny, fw, ty_h, ctas = 2000, 600, 30, 8, 444
    ntx, nty = (nx + TX - 1) // TX, (ny + ty_h - 1) // ty_h
    for order in ("row-major", "cpml-first"):
        per = [0] * ctas
        for t in range(ntx * nty):
            idx = t if order == "row-major" else cpml_first(t, ntx, nty, ty_h, nx, ny, fw, 1)
            per[t % ctas] += in_strip(idx, ntx, ty_h, nx, ny, fw, 1)
        spread = max(per) - min(per)
        assert spread <= 1 if order == "cpml-first" else spread >= 2
