"""gabe_dump.h files on the host: the reader (gabe_b200.checkpoint) takes a
dump the reference harness writes -- the reference's own step() state,
bit for bit against the golden fixture generated from the same binary --
and recognises the library's restart block, which the reference's dumps do
not carry."""
import os
import struct

import numpy as np
import pytest

from gabe_b200 import checkpoint as ck
from oracle import pyoracle as po

HERE = os.path.dirname(os.path.abspath(__file__))
REF16 = po.ref_binary(po.MODEL_LPHI4, 16, 1, 0)


@pytest.mark.skipif(not os.path.exists(REF16), reason="reference build missing (make -C oracle ref)")
def test_reads_a_dump_the_reference_harness_wrote(tmp_path):
    po.run_ref(REF16, ["--steps", "10", "--dump-at", "10", "--dump-prefix", str(tmp_path / "s")], str(tmp_path))
    path = str(tmp_path / "s10.bin")
    hd = ck.read_header(path)
    assert hd["N"] == 16 and hd["gws"] == 1 and hd["step"] == 10 and hd["L"] == 20.0 and hd["dt"] == 0.01
    st = ck.read_state(path)
    gold = np.load(os.path.join(HERE, "golden", "ref_m1_n16_g1_step10.npz"))
    for k in ("field", "dfield", "h", "l"):
        np.testing.assert_array_equal(st[k], gold[k])
    for q, name in enumerate(ck.SCALAR_NAMES):
        assert st["scalars"][name] == tuple(gold["scalars"][q])
    assert ck.read_restart_header(path) is None  # the reference writes no restart block


def test_restart_block_is_found_after_the_reference_layout_payload(tmp_path):
    cfg = po.Config(N=8, model=po.MODEL_LPHI4, gws=1)
    st = po.init_state(cfg)
    path = str(tmp_path / "d.bin")
    po.write_dump(path, st)
    assert ck.read_restart_header(path) is None
    n3, M = 8 ** 3, 8 * 8 * 5
    blk = struct.pack("<8s8iqq72x", b"GABERST1", 1, 1, 1, 0, 16, 1, 168, 4, 2 * n3 * 4, 8 * M * 4)
    with open(path, "ab") as fh:
        fh.write(blk)
    r = ck.read_restart_header(path)
    assert r == {"precision": 1, "gw_layout": 1, "expansion": 1, "tile_shape": 0, "tile_ci": 16, "e0_stale": 1,
                 "scalar_bytes": 168, "elem_bytes": 4, "field_bytes": 2 * n3 * 4, "gw_bytes": 8 * M * 4}
    back = ck.read_state(path)
    np.testing.assert_array_equal(back["field"], st.field[0])
    np.testing.assert_array_equal(back["l"], st.l[0])


def test_rejects_files_that_are_not_dumps(tmp_path):
    p = tmp_path / "x.bin"
    p.write_bytes(b"\0" * 300)
    with pytest.raises(ValueError):
        ck.read_header(str(p))


@pytest.mark.parametrize("cut", [8, 8 * 8 ** 3 * 2 + 8, 8 * 8 ** 3 * 4 + 8 * 12 * 8 * 8 * 5 + 8])
def test_truncated_dumps_name_the_short_array(tmp_path, cut):
    """A dump cut short anywhere in its payload (in field, in dfield, in l)
    is refused with the array that ran out, not read as a shorter state."""
    cfg = po.Config(N=8, model=po.MODEL_LPHI4, gws=1)
    path = str(tmp_path / "d.bin")
    po.write_dump(path, po.init_state(cfg))
    with open(path, "r+b") as fh:
        fh.truncate(256 + cut)
    which = "field" if cut < 8 * 8 ** 3 * 2 else "dfield" if cut < 8 * 8 ** 3 * 4 else "l"
    with pytest.raises(ValueError, match=f"truncated: {which} holds"):
        ck.read_state(path)
