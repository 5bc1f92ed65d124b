"""CPU: the frame-loop program's file rules (dump, src/main.cpp:680-766) with a
stand-in engine that records what it is asked to write."""
import os

import numpy as np
import pytest

from nbodysim_b200 import run
from nbodysim_b200.settings import parse_settings


class FakeEngine:
    def __init__(self):
        self.calls = []

    def save_frame(self, d, frame, binary, text, datatype_bytes):
        self.calls.append(("save", frame, binary, text, datatype_bytes))
        if binary:
            open(os.path.join(d, f"{frame:04d}.dat"), "wb").write(b"x")
        if text:
            open(os.path.join(d, f"{frame:04d}.txt"), "w").write("x")

    def render(self, **kw):
        self.calls.append(("render", kw["width"], kw["height"], kw["projection"]))
        return np.zeros((kw["height"], kw["width"], 3), np.uint8)


def settings(text):
    return parse_settings(text, warn=lambda m: None)


def test_keep_previous_rules(nb, tmp_path):
    data, img = tmp_path / "data", tmp_path / "img"
    data.mkdir(); img.mkdir()
    s = settings("dump_binary true dump_text true dump_image true keep_previous_binary false "
                 "keep_previous_text true overwrite_data true img_w 8 img_h 6 projection top")
    e = FakeEngine()
    for f in range(3):
        run.dump(e, s, f, str(data), str(img), 8)
    assert sorted(os.listdir(data)) == ["0000.txt", "0001.txt", "0002.dat", "0002.txt"]
    assert sorted(os.listdir(img)) == ["0000.ppm", "0001.ppm", "0002.ppm"]
    assert e.calls[0] == ("save", 0, True, True, 8) and e.calls[1] == ("render", 8, 6, 2)
    body = (img / "0002.ppm").read_bytes()
    assert body.startswith(b"P6\n8 6\n255\n") and len(body) == len(b"P6\n8 6\n255\n") + 8 * 6 * 3


def test_overwrite_disabled_aborts(nb, tmp_path):
    data, img = tmp_path / "data", tmp_path / "img"
    data.mkdir(); img.mkdir()
    (data / "0005.dat").write_bytes(b"old")
    s = settings("dump_binary true dump_text false dump_image false overwrite_data false")
    with pytest.raises(SystemExit) as ex:
        run.dump(FakeEngine(), s, 5, str(data), str(img), 8)
    assert ex.value.code == 1 and (data / "0005.dat").read_bytes() == b"old"
    s = settings("dump_binary true dump_text false dump_image false overwrite_data true")
    e = FakeEngine()
    run.dump(e, s, 5, str(data), str(img), 4)
    assert e.calls == [("save", 5, True, False, 4)] and (data / "0005.dat").read_bytes() == b"x"
