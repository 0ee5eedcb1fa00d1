"""The run-time kernel configuration table (rocsolver_b200_tuning_*): parsing, round trip,
rejection of malformed text, loading from a file.  Host-only: no kernel runs."""
import rocsolver_b200 as rs

SUCCESS, INVALID_POINTER, INVALID_VALUE = 0, 3, 11


def _restore(text):
    assert rs.set_tuning_table(text) == SUCCESS


def test_roundtrip_sorted_and_comments():
    old = rs.tuning_table()
    try:
        text = ("# comment line\n"
                "vbatched d 512 256 2 16 64 1 0\n"
                "getrf d 256 256 1 32 64 0   # trailing comment\n"
                "getrf d 128 128 1 32 0 1\n"
                "getrf t 512 256 2 32 128 1\n"
                "getrf s 256 128 2 32 96 1\n")
        assert rs.set_tuning_table(text) == SUCCESS
        got = rs.tuning_table().splitlines()
        assert got == ["getrf d 128 128 1 32 0 1",
                       "getrf d 256 256 1 32 64 0",
                       "getrf s 256 128 2 32 96 1",
                       "getrf t 512 256 2 32 128 1",
                       "vbatched d 512 256 2 16 64 1 0"]
    finally:
        _restore(old)


def test_malformed_text_is_rejected_and_table_kept():
    old = rs.tuning_table()
    try:
        assert rs.set_tuning_table("getrf d 256 256 1 32 64 0\n") == SUCCESS
        for bad in ("getrf x 256 256 1 32 64 0", "getrf d 256 256 1 32 64",
                    "getrf d 256 256 1 32 64 0 9", "potrf d 64 1 2 3 4 5",
                    "getrf d 0 256 1 32 64 0", "getrf d 256 -1 1 32 64 0",
                    "vbatched d 512 256 2 16 64 1", "vbatched t 512 256 2 16 64 1 0"):
            assert rs.set_tuning_table(bad) == INVALID_VALUE, bad
            assert rs.tuning_table() == "getrf d 256 256 1 32 64 0\n"
        assert rs.lib().rocsolver_b200_tuning_set(None) == INVALID_POINTER
        assert rs.set_tuning_table("") == SUCCESS
        assert rs.tuning_table() == ""
    finally:
        _restore(old)


def test_load_from_file(tmp_path):
    old = rs.tuning_table()
    try:
        f = tmp_path / "t.txt"
        f.write_text("getrf s 512 256 2 16 128 0\n")
        assert rs.lib().rocsolver_b200_tuning_load(str(f).encode()) == SUCCESS
        assert rs.tuning_table() == "getrf s 512 256 2 16 128 0\n"
        assert rs.lib().rocsolver_b200_tuning_load(str(tmp_path / "missing").encode()) \
            == INVALID_VALUE
    finally:
        _restore(old)


def test_get_truncates_to_buffer():
    import ctypes
    old = rs.tuning_table()
    try:
        assert rs.set_tuning_table("getrf d 256 256 1 32 64 0\n") == SUCCESS
        buf = ctypes.create_string_buffer(8)
        full = rs.lib().rocsolver_b200_tuning_get(buf, 8)
        assert full == len("getrf d 256 256 1 32 64 0\n") + 1
        assert buf.value == b"getrf d"
    finally:
        _restore(old)
