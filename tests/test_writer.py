"""output_potential (bit_write_potential) byte for byte against a file the reference's own
output_potential wrote (tests/golden/output_potential.txt).  Host code: no GPU."""
import os

from conftest import GOLDEN, load_golden


def test_writer_matches_reference_output_byte_for_byte(tmp_path):
    import bit_b200 as B
    g = load_golden("output_potential")
    out = tmp_path / "pot.txt"
    B.write_potential(str(out), g["x"], g["y"], g["z"], g["pot"])
    ref = open(os.path.join(GOLDEN, "output_potential.txt"), "rb").read()
    assert out.read_bytes() == ref
