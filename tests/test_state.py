"""State files: the checkpoint / interchange format."""
import numpy as np
import pytest

from cosmograph_b200 import ics, state as S


def test_roundtrip(tmp_path):
    st = ics.perturbed((5, 6, 7), S.DUST, seed=2)
    st.step, st.frw_phi, st.frw_K, st.fluids = 3, 0.1, -2.5, ((0.2, 0.0), (0.1, 1.0 / 3.0))
    st.save(tmp_path / "a.bin")
    back = S.load(tmp_path / "a.bin")
    assert np.array_equal(back.fields, st.fields)
    assert (back.step, back.frw_phi, back.frw_K, back.fluids, back.lam) == \
        (st.step, st.frw_phi, st.frw_K, st.fluids, st.lam)
    assert back.names == S.BSSN_FIELDS + S.DUST_FIELDS


def test_truncated_and_foreign_files_are_rejected(tmp_path):
    st = ics.perturbed((4, 4, 4), S.SCALAR)
    p = tmp_path / "s.bin"
    st.save(p)
    raw = p.read_bytes()
    (tmp_path / "t.bin").write_bytes(raw[:-8])
    with pytest.raises(ValueError, match="truncated"):
        S.load(tmp_path / "t.bin")
    (tmp_path / "m.bin").write_bytes(b"NOTSTATE" + raw[8:])
    with pytest.raises(ValueError, match="not a state"):
        S.load(tmp_path / "m.bin")
    with pytest.raises(ValueError):
        S.BoxState(fields=np.zeros((3, 4, 4, 4)), matter=S.DUST, dx=0.1, dt=0.01).save(tmp_path / "x.bin")


def test_field_counts():
    assert [S.num_fields(m) for m in (S.VACUUM, S.DUST, S.SCALAR)] == [18, 22, 23]
