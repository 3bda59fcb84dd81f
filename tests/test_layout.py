"""The record slot layout of the wavefront passes, checked on the host (no
GPU): a slot is CR_N = 16 words (the 11-word record and MR) and its 16-byte
vectors are stored in an order rotated by the slot's position t in its step
block (rec_vec_pos).  The residual kernel stores with t = slot mod 8, the
passes load with t = their thread index, so the two must agree on t mod 8.
In every phase of eight lanes of a 16-byte shared-memory load, the lanes'
vectors must land on eight different 16-byte bank groups."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


@pytest.fixture(scope="module")
def layout(tmp_path_factory):
    if not os.path.exists(NVCC) and shutil.which("nvcc") is None:
        pytest.skip("nvcc not present")
    exe = tmp_path_factory.mktemp("layout") / "layout_probe"
    subprocess.run([NVCC, "-std=c++17", "-I", os.path.join(REPO, "cgli_fu_flow_b200", "csrc"),
                    os.path.join(HERE, "csrc", "layout_probe.cu"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    pos = {"d": {}, "f": {}}
    info = {}
    for line in out.splitlines():
        f = line.split()
        if f[0] in pos:
            pos[f[0]][(int(f[1]), int(f[2]))] = int(f[3])
        else:
            info[f[0]] = [int(x) for x in f[1:]]
    return pos, info


def test_slot_is_sixteen_words(layout):
    _, info = layout
    assert info["slot"] == [16, 11]


@pytest.mark.parametrize("kind,nvec,slot_bytes", [("d", 8, 128), ("f", 4, 64)])
def test_vector_rotation_is_a_conflict_free_permutation(layout, kind, nvec, slot_bytes):
    pos, _ = layout
    p = pos[kind]
    for t in range(256):
        assert sorted(p[(t, u)] for u in range(nvec)) == list(range(nvec))   # a permutation of the slot
        for u in range(nvec):
            assert p[(t, u)] == p[(t % 8, u)]                                # writer and reader agree on t mod 8
    for base in range(0, 256, 8):                                          # one phase of eight lanes
        for u in range(nvec):
            groups = [((t * slot_bytes) // 16 + p[(t, u)]) % 8 for t in range(base, base + 8)]
            assert len(set(groups)) == 8, (kind, base, u, groups)


def test_step_blocks_hold_a_whole_number_of_rotations(layout):
    # the writer's t = slot mod 8 equals the position in the step block only
    # if every step block starts at a multiple of 8 slots
    _, info = layout
    ti, tj, tif, tjf = info["tile"]
    assert (ti * tj) % 8 == 0 and (tif * tjf) % 8 == 0
