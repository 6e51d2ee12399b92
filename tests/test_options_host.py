"""cgb_set_option / cgb_get_option on the host (no GPU needed): every speed knob takes the
values its documentation names, refuses the values around them with a message naming the
option, and reads back what was set; unknown names are refused."""
import pytest

from cablegen_b200 import _lib

# option: (accepted values, refused values, default)
KNOBS = {
    "index": ([0, 1, 2], [-1, 3], 2),
    "solve_variant": ([0, 1], [-1, 2], 1),
    "sort_variant": ([0, 1, 2, 3, 4, 5], [-1, 6], 4),
    "hash_load_pct": ([0, 10, 25, 45, 90], [-1, 5, 9, 91], 0),
    "region_build": ([0, 1], [-1, 2], 1),
    "move_window": ([1, 2, 3, 4], [0, 5], 1),
    "hash_compact": ([0, 1], [-1, 2], 1),
    "fp64_top_layers": ([0, 4, 100000], [-1, 100001], 4),
    "bucket_bits": ([0, 16, 30], [-1, 31], None),
}


@pytest.fixture(scope="module")
def L():
    return _lib.lib()


def get(L, name):
    return L.cgb_get_option(name.encode())


def set_(L, name, value):
    return L.cgb_set_option(name.encode(), value)


@pytest.mark.parametrize("name", sorted(KNOBS))
def test_knob_range(L, name):
    ok, bad, default = KNOBS[name]
    old = get(L, name)
    if default is not None:
        assert old == default, name
    try:
        for v in ok:
            assert set_(L, name, v) == 0, (name, v)
            assert get(L, name) == v, (name, v)
        last = get(L, name)
        for v in bad:
            assert set_(L, name, v) == -1, (name, v)
            assert name in L.cgb_last_error().decode(), (name, v)
            assert get(L, name) == last, (name, v)  # a refused value changes nothing
    finally:
        assert set_(L, name, old) == 0


def test_unknown_option(L):
    assert set_(L, "no_such_option", 1) == -1
    assert "unknown option" in L.cgb_last_error().decode()
    assert get(L, "no_such_option") == -1
