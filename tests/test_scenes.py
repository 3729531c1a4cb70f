import numpy as np

from ipc_warp_b200 import scenes


def test_cube_counts_match_config():
    sc = scenes.two_cubes()
    assert sc.n_verts == 2 * 729 and sc.tets.shape[0] == 2 * 2560 and sc.n_tris == 2 * 768
    assert sc.n_edges == 2304


def test_rod_counts_match_config():
    m = scenes.hex_grid_tets(4, 4, 256, (0.1, 0.1, 6.4))
    assert m.x.shape[0] == 6425 and m.tets.shape[0] == 20480 and m.triangles.shape[0] == 8256


def test_surface_is_closed_and_outward():
    m = scenes.hex_grid_tets(3, 4, 5, (1.0, 2.0, 3.0))
    x, t = m.x, m.triangles
    vol = np.einsum("ij,ij->i", x[t[:, 0]], np.cross(x[t[:, 1]], x[t[:, 2]])).sum() / 6
    assert abs(vol - 6.0) < 1e-12
    assert m.edges.shape[0] * 2 == t.shape[0] * 3
