"""The .prm format and the factory's name rule."""
import pytest

from listctrecons_b200 import FileParams, ParameterError, ReconstrctorAbstractFactory
from listctrecons_b200.recon import FDKReconstructor


def test_roundtrip_and_alias(tmp_path, small_geo):
    fp = small_geo.file_params(str(tmp_path), str(tmp_path))
    fp.write(tmp_path / "a.prm")
    back = FileParams.read(tmp_path / "a.prm")
    assert back == fp
    txt = (tmp_path / "a.prm").read_text().replace("PitchValue:", "TableFeed:")
    (tmp_path / "b.prm").write_text(txt)
    assert FileParams.read(tmp_path / "b.prm").PitchValue == fp.PitchValue


def test_missing_key_reports_first_missing(tmp_path, small_geo):
    fp = small_geo.file_params(str(tmp_path), str(tmp_path))
    fp.write(tmp_path / "a.prm")
    lines = [l for l in (tmp_path / "a.prm").read_text().splitlines() if not l.startswith("Dz:")]
    (tmp_path / "c.prm").write_text("\n".join(lines))
    with pytest.raises(ParameterError, match="Parameter not found in prm file:Dz"):
        FileParams.read(tmp_path / "c.prm")
    with pytest.raises(ParameterError, match="Parameter file not found"):
        FileParams.read(tmp_path / "nope.prm")


def test_factory_name_rule():
    fac = ReconstrctorAbstractFactory()
    # str.find("fdk") is truthy unless "fdk" starts the name (Src/ReconstructorAbstractFactory.cpp:13)
    assert isinstance(fac.createReconstructor("Helicalfdkramprebingpu"), FDKReconstructor)
    assert isinstance(fac.createReconstructor("anything"), FDKReconstructor)
    with pytest.raises(ValueError):
        fac.createReconstructor("fdkHelical")
