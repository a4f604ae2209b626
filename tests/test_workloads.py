"""Seeded synthetic structures and path lists."""
import numpy as np

from feffgpu_b200 import workloads as W


def test_random_packing_and_paths():
    pos, lab, box = W.random_packing(400, 0.08, 1.8, seed=3)
    d = pos[:, None] - pos[None]
    d -= box * np.round(d / box)
    r = np.sqrt((d ** 2).sum(-1)) + np.eye(len(pos)) * 99
    assert r.min() >= 1.8 - 1e-9
    assert abs(box - (400 / 0.08) ** (1 / 3)) < 1e-12
    ab = int(W.central_atom(pos, box, lab, "Fe", 1)[0])
    ipot_of = np.array([{"Fe": 1, "O": 2, "Pt": 3}[x] for x in lab])
    paths = W.random_paths(pos, box, ab, {2: 5, 3: 20, 4: 30}, rmax=6.0, seed=1, ipot_of=ipot_of)
    for nleg, (c, ip, atoms) in paths.items():
        assert c.shape == (len(atoms), nleg, 3) and np.all(c[:, 0] == 0) and np.all(ip[:, 0] == 0)
        legs = np.linalg.norm(np.diff(np.concatenate([c, c[:, :1]], 1), axis=1), axis=-1)
        assert np.all(legs.sum(1) / 2 <= 6.0 + 1e-9) and np.all(legs <= 6.0 + 1e-9) and np.all(legs > 1.0)
        assert np.all(atoms[:, -1] != ab)
        assert np.all(ip[:, 1:][atoms != ab] == ipot_of[atoms[atoms != ab]])


def test_lattices():
    pts = W.fcc_cluster(3.61, 6.0)
    assert np.all(pts[0] == 0) and len(pts) == 79
    p, box = W.bcc_supercell(4, 2.87)
    assert len(p) == 128 and box == 4 * 2.87
    p, lab, box = W.rock_salt_supercell(2, 4.177)
    assert len(p) == 64 and (lab == "Ni").sum() == 32


def test_md_batch_paths_of_bcc():
    """Every 2- and 3-leg bcc path within 5.5 A (58 + 384 per absorber), exact lattice offsets without disorder,
    deg = 1 / absorbers and one row per frame."""
    s = W.bcc_site_paths(16, 2.87, 5.5)
    assert len(s[2]) == 58 and len(s[3]) == 384
    a = 2.87 / 2
    r = np.linalg.norm(s[3] * a, axis=2)
    d = np.linalg.norm((s[3][:, 1] - s[3][:, 0]) * a, axis=1)
    assert np.all(r.sum(1) + d <= 11.0 + 1e-9) and np.all(d > 0)
    groups, per = W.md_batch(frames=3, absorbers=4, sigma=0.0, seed=1)
    assert per == 442
    for (c, ip, deg, row), nleg in zip(groups, (2, 3)):
        assert c.shape == (3 * 4 * len(s[nleg]), nleg, 3)
        assert np.allclose(c[: 4 * len(s[nleg]), 1:].reshape(4, -1, nleg - 1, 3), s[nleg][None] * a, atol=1e-12)
        assert np.all(ip[:, 0] == 0) and np.all(ip[:, 1:] == 1)
        assert np.allclose(deg, 0.25) and sorted(set(row.tolist())) == [0, 1, 2]
