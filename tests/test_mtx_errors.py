"""Matrix Market reader failure handling (host code, no GPU): malformed
files are reported with a status and a message, never a crash."""
import pytest


@pytest.mark.parametrize("text", [
    "",                                                                  # empty
    "not a matrix market file\n1 1 1\n1 1 1.0\n",                        # bad banner
    "%%MatrixMarket matrix coordinate real general\n3 3\n",              # short size line
    "%%MatrixMarket matrix coordinate real general\n3 3 2\n1 1 1.0\n",   # fewer entries than declared
    "%%MatrixMarket matrix coordinate real general\n3 3 1\n4 1 1.0\n",   # row out of range
    "%%MatrixMarket matrix coordinate real general\n3 3 1\n1 0 1.0\n",   # column out of range
    "%%MatrixMarket matrix coordinate real general\n3 3 1\n1 1 abc\n",   # bad value
])
def test_malformed_files_rejected(mf, tmp_path, text):
    f = tmp_path / "bad.mtx"
    f.write_text(text)
    with pytest.raises(mf.MfError):
        mf.read_matrix_market(f)


def test_missing_file_rejected(mf, tmp_path):
    with pytest.raises(mf.MfError):
        mf.read_matrix_market(tmp_path / "none.mtx")
