"""Wire format of the slice service (net.py): the same payloads as the reference's own
send() (golden fixtures made by running it), receive into reused host buffers, the BF16
reply encoding and the geometry messages. CPU only; the server is tested on the GPU."""
import threading
from multiprocessing import Pipe

import numpy as np
import pytest
import torch

from conftest import golden
from tomography_local_demo_b200 import ParallelGeometry, circular_cone_vectors
from tomography_local_demo_b200 import net


class _Recorder:
    def __init__(self):
        self.payloads = []

    def send_bytes(self, b):
        self.payloads.append(bytes(b))


class _Replay:
    """A connection that hands back recorded payloads (recv_bytes / recv_bytes_into)."""

    def __init__(self, payloads):
        self.payloads = list(payloads)

    def recv_bytes(self):
        return self.payloads.pop(0)

    def recv_bytes_into(self, buf):
        b = self.payloads.pop(0)
        memoryview(buf)[:len(b)] = b
        return len(b)


def _messages():
    rng = np.random.default_rng(11)
    return [({"cmd": "hello", "role": "adapter"}, None),
            ({"cmd": "projections", "indices": [3, 1, 2]}, rng.normal(size=(4, 3, 5)).astype(np.float32)),
            ({"version": 7}, rng.normal(size=(6, 6)).astype(np.float32)),
            ({"origin": [0.5, -1.0, 2.0], "spacing": 0.25}, rng.gamma(2.0, 1.0, (2, 3, 4)).astype(np.float32)),
            ({"cmd": "raw", "note": "u16"}, rng.integers(0, 65535, (2, 3, 4)).astype(np.uint16)),
            ({"cmd": "slice", "origin": [0.0, 0.0, 0.0], "normal": [0.0, 0.0, 1.0], "n": 64, "zoom": 1.0,
              "center": None}, None)]


def test_send_writes_the_reference_payloads():
    g = golden("net_frames.npz")
    for i, (h, arr) in enumerate(_messages()):
        rec = _Recorder()
        net.send(rec, h, arr)
        want = [g[f"m{i}_p{j}"].tobytes() for j in range(int(g[f"m{i}_count"]))]
        assert rec.payloads == want


@pytest.mark.parametrize("frames", [None, "pool"])
def test_recv_reads_the_reference_payloads(frames):
    g = golden("net_frames.npz")
    pool = net.PinnedFrames(pinned=False) if frames else None
    for i, (h, arr) in enumerate(_messages()):
        conn = _Replay([g[f"m{i}_p{j}"].tobytes() for j in range(int(g[f"m{i}_count"]))])
        hr, ar = net.recv(conn, pool)
        assert hr == h
        if arr is None:
            assert ar is None
            continue
        got = ar.numpy() if isinstance(ar, torch.Tensor) else ar
        np.testing.assert_array_equal(got.view(arr.dtype), arr)
        if pool is not None:
            pool.release(ar)


def test_geometry_messages_match_the_reference_and_round_trip():
    g = golden("net_frames.npz")
    cone = circular_cone_vectors(12, 300.0, 600.0, 8, 10, 1.5, det_shift_u=0.7)
    par = ParallelGeometry(np.linspace(0, np.pi, 9, endpoint=False), 6, 7, 0.5, 0.25)
    for tag, geom in (("cone", cone), ("par", par)):
        rec = _Recorder()
        net.send(rec, *net.geometry_message(geom))
        assert rec.payloads == [g[f"geom_{tag}_p0"].tobytes(), g[f"geom_{tag}_p1"].tobytes()]
        h, arr = net.recv(_Replay(rec.payloads))
        back = net.geometry_from_message(h, arr)
        assert type(back) is type(geom) and (back.rows, back.cols) == (geom.rows, geom.cols)
        np.testing.assert_array_equal(back.volume_box(), geom.volume_box())
        if tag == "cone":
            np.testing.assert_array_equal(back.vectors, geom.vectors)
            assert back.angular_range == geom.angular_range
        else:
            np.testing.assert_array_equal(back.angles, geom.angles)
            assert (back.pixel_u, back.pixel_v) == (geom.pixel_u, geom.pixel_v)


def test_framing_over_a_pipe_reuses_buffers_and_refuses_non_numbers():
    a, b = Pipe()
    pool = net.PinnedFrames(pinned=False)
    rng = np.random.default_rng(2)
    arrays = [rng.normal(size=(3, 7)).astype(np.float64), rng.integers(0, 9, (5,)).astype(np.int32),
              np.zeros((0, 4), np.float32), rng.normal(size=(2, 2)).astype(np.float32),
              rng.integers(0, 65535, (3, 384, 486)).astype(np.uint16)]    # > 16 KiB: header, then payload

    def writer():
        for k, arr in enumerate(arrays):
            net.send(a, {"k": k}, arr)

    t = threading.Thread(target=writer)
    t.start()
    for k, arr in enumerate(arrays):
        h, got = net.recv(b, pool)
        assert h == {"k": k}
        np.testing.assert_array_equal(got.numpy().view(arr.dtype), arr)
        pool.release(got)
    t.join()
    assert len(pool._free) <= 3                       # buffers went back and were reused
    a.send_bytes(b'{"_array": {"dtype": "|O", "shape": [1]}}')
    with pytest.raises(ValueError):
        net.recv(b)
    a.send_bytes(b'{"_array": {"dtype": "<f4", "shape": [4]}}')
    a.send_bytes(b"\x00" * 12)                        # 3 floats where 4 were announced
    with pytest.raises(ValueError):
        net.recv(b, pool)
    for shape in ([-1, 4], [1 << 20, 1 << 20]):       # negative / beyond the payload limit
        a.send_bytes(('{"_array": {"dtype": "<f4", "shape": %s}}' % shape).encode())
        with pytest.raises(ValueError):
            net.recv(b, pool)
    small = net.PinnedFrames(pinned=False, keep_bytes=8)
    small.release(small.take(64))                     # above keep_bytes: not kept
    small.release(small.take(8))
    assert [t.numel() for t, _ in small._free] == [8]


def test_bf16_replies_round_to_nearest_even():
    rng = np.random.default_rng(4)
    img = np.concatenate([rng.normal(size=1000) * 10.0 ** rng.uniform(-8, 8, 1000),
                          [0.0, -0.0, 1.0, -2.5, np.inf, -np.inf]]).astype(np.float32)
    # values exactly between two BF16 neighbours: ties go to the even mantissa
    ties = (np.array([0x3F808000, 0x3F818000, 0xBF808000], np.uint32)).view(np.float32)
    img = np.concatenate([img, ties])
    data, extra = net.encode_image(img, "bf16")
    assert extra == {"encoding": "bf16"} and data.dtype == np.uint16
    bits = img.view(np.uint32).astype(np.uint64)
    want = ((bits + 0x7FFF + ((bits >> 16) & 1)) >> 16).astype(np.uint16)
    np.testing.assert_array_equal(data, want)
    back = net.decode_image(extra, data)
    np.testing.assert_array_equal(back, (want.astype(np.uint32) << 16).view(np.float32))
    fin = np.isfinite(img) & (img != 0)
    assert np.all(np.abs(back[fin] - img[fin]) <= np.abs(img[fin]) * 2.0 ** -8)
    f32, extra32 = net.encode_image(img, "f32")
    assert extra32 == {} and f32.dtype == np.float32
    with pytest.raises(ValueError):
        net.encode_image(img, "f8")


def test_parse_address():
    assert net.parse_address("gpu-host:6000") == ("gpu-host", 6000)
    assert net.parse_address(":6001") == ("127.0.0.1", 6001)
    assert net.parse_address("localhost:") == ("localhost", net.DEFAULT_PORT)
