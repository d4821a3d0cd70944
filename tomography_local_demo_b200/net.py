"""Wire-compatible slice service (the client/server split of minirecast net.py:1-270):
an adapter pushes a scan's geometry and projections, viewers ask for slices, previews
and COR changes, and the server does all reconstruction on its GPU.

The message layout is the reference's (net.py:40-59), so the reference's adapters and
viewers can talk to this server and these clients to the reference's server: one message
with a UTF-8 JSON header and, when the header's "_array" entry names a dtype and a shape,
one more message with the array's raw bytes (numbers only - nothing is unpickled).
Connections are `multiprocessing.connection` ones, authenticated (HMAC) with the shared
key in $MINIRECAST_KEY.

Beyond the reference:
* receive side: array payloads are read from the connection's descriptor straight into
  page-locked buffers of a reused pool (`PinnedFrames`) and handed to the reconstructor as
  pinned tensors, so projections go socket -> page-locked memory -> device with no
  intermediate host copy (the standard `recv_bytes` / `recv_bytes_into` read into a
  BytesIO and copy);
* "raw_projections" (uint16 counts [k, R0, C0] through the fused ingest) and "flat_dark"
  (`set_flat_dark`, flat and dark stacked as [2, n, R0, C0]) commands;
* "slice" and "slices" take "encoding": "bf16": the reply carries each FP32 value rounded
  to nearest-even BF16 as uint16 (half the bytes; the reference's `recv` accepts it as an
  integer array) and says so in the header; `decode_image` widens it back;
* "slices" answers several slice requests with one array; "reset" starts a new scan with
  the same geometry;
* slices and previews are answered by the continuously batched `SliceServer`.
"""
import json
import os
import struct
import threading
import time
from multiprocessing.connection import Client, Connection, Listener

import numpy as np
import torch

from .geometry import ConeVecGeometry, ParallelGeometry
from .recon import SliceReconstructor, plane_size_for_box, slice_points
from .server import SliceServer

DEFAULT_PORT = 5558
MAX_ARRAY_BYTES = 1 << 36           # largest array payload accepted (64 GiB)


def authkey():
    """The shared connection key (net.py:29-30): $MINIRECAST_KEY, else the demo key."""
    return os.environ.get("MINIRECAST_KEY", "minirecast-demo").encode()


def parse_address(text):
    """"host:port", ":port" or "host:" -> (host, port) (net.py:33-35)."""
    host, _, port = str(text).rpartition(":")
    return (host if host else "127.0.0.1", int(port) if port else DEFAULT_PORT)


# ------------------------------------------------------------------ framing
def _array_spec(header):
    """(dtype, shape) of the array announced by a header, or None; numbers only."""
    spec = header.pop("_array", None)
    if spec is None:
        return None
    dtype = np.dtype(spec["dtype"])
    if dtype.kind not in ("f", "i", "u"):
        raise ValueError(f"refusing array dtype {dtype}")
    return dtype, tuple(int(s) for s in spec["shape"])


def send(conn, header, array=None):
    """Send a header (dict) and an optional array (net.py:40-48 layout)."""
    out = dict(header)
    if array is not None:
        if isinstance(array, torch.Tensor):
            array = array.detach().cpu().numpy()
        array = np.ascontiguousarray(array)
        out["_array"] = {"dtype": array.dtype.str, "shape": list(array.shape)}
    conn.send_bytes(json.dumps(out).encode())
    if array is not None:
        conn.send_bytes(array.reshape(-1).view(np.uint8))       # the array's bytes, no copy


def recv(conn, frames=None):
    """Receive (header, array or None) (net.py:51-59 layout). With `frames` (a
    PinnedFrames pool) the array bytes land in a page-locked buffer and the array comes
    back as a pinned torch tensor viewing it (release it with frames.release after the
    device copies that read it are queued); otherwise as a NumPy array."""
    header = json.loads(conn.recv_bytes().decode())
    spec = _array_spec(header)
    if spec is None:
        return header, None
    dtype, shape = spec
    nbytes = int(np.prod(shape, dtype=np.int64)) * dtype.itemsize
    if any(d < 0 for d in shape) or nbytes > MAX_ARRAY_BYTES:
        raise ValueError(f"refusing an array of shape {shape} ({nbytes} bytes)")
    if frames is None or not dtype.isnative:
        data = conn.recv_bytes()
        if len(data) != nbytes:
            raise ValueError(f"array message of {len(data)} bytes, header announced {nbytes}")
        return header, np.frombuffer(data, dtype=dtype).reshape(shape)
    buf = frames.take(max(nbytes, 1))
    got = _recv_bytes_into(conn, memoryview(buf.numpy()))
    if got != nbytes:
        frames.release(buf)
        raise ValueError(f"array message of {got} bytes, header announced {nbytes}")
    return header, frames.lend(buf, buf[:nbytes].view(_TORCH_DTYPE[dtype]).view(shape))


def _read_exact(fd, view):
    """Fill `view` from file descriptor `fd` (EOFError if the peer closes first)."""
    got = 0
    while got < len(view):
        n = os.readv(fd, [view[got:]])
        if n == 0:
            raise EOFError("connection closed inside a message")
        got += n


def _recv_bytes_into(conn, view):
    """conn.recv_bytes_into(view) without the intermediate copy: on a POSIX socket or pipe
    Connection the message's length prefix (4 bytes big-endian, or -1 then 8 bytes for
    messages over 2 GiB - multiprocessing.connection's framing) is read first and the
    payload is read from the descriptor straight into `view`. Other connections use
    recv_bytes_into, which reads the message into a BytesIO and copies it."""
    if os.name != "posix" or not isinstance(conn, Connection):
        return conn.recv_bytes_into(view)
    fd = conn.fileno()
    head = bytearray(4)
    _read_exact(fd, memoryview(head))
    size = struct.unpack("!i", head)[0]
    if size == -1:
        head = bytearray(8)
        _read_exact(fd, memoryview(head))
        size = struct.unpack("!Q", head)[0]
    if size > len(view):
        raise ValueError(f"array message of {size} bytes does not fit its {len(view)}-byte buffer")
    _read_exact(fd, view[:size])
    return size


_TORCH_DTYPE = {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
                np.dtype(np.float16): torch.float16, np.dtype(np.uint8): torch.uint8,
                np.dtype(np.int8): torch.int8, np.dtype(np.int16): torch.int16,
                np.dtype(np.uint16): torch.int16, np.dtype(np.int32): torch.int32,
                np.dtype(np.uint32): torch.int32, np.dtype(np.int64): torch.int64,
                np.dtype(np.uint64): torch.int64}


class PinnedFrames:
    """Reusable page-locked receive buffers. `take(n)` returns a uint8 tensor of at least
    n bytes whose previous contents are no longer read by any queued device copy;
    `release(buf, streams)` returns it to the pool once the copies queued on `streams`
    so far have run. Buffers grow to the largest payload seen; one larger than `keep_bytes`
    is not kept (torch's host cache holds it until the copies that read it have run).
    `pinned=False` gives ordinary host memory (no CUDA needed)."""

    def __init__(self, pinned=True, keep_bytes=1 << 30):
        self.pinned = pinned and torch.cuda.is_available()
        self.keep_bytes = int(keep_bytes)
        self._free = []                 # [(uint8 buffer, [events])]
        self._lent = {}                 # data pointer of a lent view -> its uint8 buffer
        self._lock = threading.Lock()

    def take(self, nbytes):
        with self._lock:
            best = None
            for k, (t, _) in enumerate(self._free):
                if t.numel() >= nbytes and (best is None or t.numel() < self._free[best][0].numel()):
                    best = k
            if best is not None:
                t, events = self._free.pop(best)
                for ev in events:
                    ev.synchronize()
                return t
        t = torch.empty(int(nbytes), dtype=torch.uint8)
        return t.pin_memory() if self.pinned else t

    def lend(self, buf, view):
        """Remember that `view` (which starts at buf's first byte) belongs to `buf`."""
        with self._lock:
            self._lent[view.data_ptr()] = buf
        return view

    def release(self, buf, streams=()):
        """Return a buffer, or an array that recv() lent from one, to the pool."""
        with self._lock:
            base = self._lent.pop(buf.data_ptr(), buf)
        if base.numel() > self.keep_bytes:
            return
        events = []
        for st in streams:
            ev = torch.cuda.Event()
            ev.record(st)
            events.append(ev)
        with self._lock:
            self._free.append((base, events))


# ------------------------------------------------------------------ payload helpers
def geometry_message(geom):
    """(header, array) describing a geometry (net.py:62-73 fields)."""
    box = [float(b) for b in geom.volume_box()]
    if isinstance(geom, ParallelGeometry):
        h = dict(cmd="geometry", kind="parallel", rows=geom.rows, cols=geom.cols,
                 pixel_u=geom.pixel_u, pixel_v=geom.pixel_v, box=box)
        return h, np.asarray(geom.angles, dtype=np.float64)
    h = dict(cmd="geometry", kind="cone", rows=geom.rows, cols=geom.cols,
             angular_range=float(geom.angular_range), box=box)
    return h, np.asarray(geom.vectors, dtype=np.float64)


def geometry_from_message(h, arr):
    """The geometry a "geometry" message describes (net.py:76-83)."""
    arr = np.asarray(arr, dtype=np.float64)
    box = np.asarray(h["box"], dtype=np.float64)
    if h["kind"] == "parallel":
        return ParallelGeometry(arr, int(h["rows"]), int(h["cols"]), float(h["pixel_u"]),
                                float(h["pixel_v"]), box=box)
    return ConeVecGeometry(arr.reshape(-1, 12), int(h["rows"]), int(h["cols"]),
                           float(h["angular_range"]), box=box)


def encode_image(img, encoding="f32"):
    """(array, header fields) of an FP32 image for a reply: "f32" as is, "bf16" rounded to
    nearest-even BF16 and carried as uint16 bits."""
    if encoding in (None, "f32"):
        return np.ascontiguousarray(img, dtype=np.float32), {}
    if encoding != "bf16":
        raise ValueError(f"unknown encoding {encoding!r}")
    t = torch.from_numpy(np.ascontiguousarray(img, dtype=np.float32)).to(torch.bfloat16)
    return t.view(torch.int16).numpy().view(np.uint16), {"encoding": "bf16"}


def decode_image(header, arr):
    """An image reply as float32 (widens "bf16" replies)."""
    arr = np.asarray(arr)
    if header.get("encoding") == "bf16":
        return (arr.astype(np.uint32) << 16).view(np.float32)
    return arr.astype(np.float32, copy=False)


# ------------------------------------------------------------------ server
class Server:
    """The reference's server (net.py:87-178) on this package's reconstructor: same
    commands and replies, plus the extensions in the module docstring. One thread per
    connection; the reconstructor and its SliceServer are replaced by each "geometry"."""

    def __init__(self, host="127.0.0.1", port=DEFAULT_PORT, window="shepp-logan", backend="auto",
                 gaussian=0.0, tilt=0.0, verbose=True, store="fp32", filter="fft",
                 budget_bytes=4e9, device=None):
        self.address = (host, port)
        self.verbose = verbose
        self.opts = dict(window=window, backend=backend, gaussian=gaussian, tilt=tilt, store=store,
                         filter=filter, device=device)
        self.budget = budget_bytes
        self.recon = None
        self.slices = None
        self.frames = PinnedFrames()
        self.lock = threading.Lock()
        self._listener = None

    def log(self, msg):
        if self.verbose:
            print(msg, flush=True)

    def listen(self):
        """Bind the listener (port 0 picks a free port) and return the bound address."""
        if self._listener is None:
            self._listener = Listener(self.address, authkey=authkey())
            self.address = self._listener.address
        return self.address

    def serve_forever(self):
        self.listen()
        self.log(f"[server] listening on {self.address[0]}:{self.address[1]}")
        while True:
            try:
                conn = self._listener.accept()
            except OSError:
                if self._listener is None:
                    return                           # closed
                continue
            except Exception as e:                   # bad key, port scan, ...
                self.log(f"[server] rejected connection: {e}")
                continue
            threading.Thread(target=self.serve_connection, args=(conn,), daemon=True).start()

    def close(self):
        lst, self._listener = self._listener, None
        if lst is not None:
            lst.close()
        with self.lock:
            if self.slices is not None:
                self.slices.close()
                self.slices = None

    def _current(self):
        with self.lock:
            if self.recon is None:
                raise RuntimeError("no scan yet - start an adapter (minirecast push ...)")
            return self.recon, self.slices

    def _new_scan(self, geom):
        rec = SliceReconstructor(None, geom, verbose=False, **self.opts)
        srv = SliceServer(rec, budget_bytes=self.budget)
        with self.lock:
            old, self.recon, self.slices = self.slices, rec, srv
        if old is not None:
            old.close()
        return rec

    def _release(self, arr, rec):
        if isinstance(arr, torch.Tensor):
            self.frames.release(arr, (rec.ingest_stream, rec.copy_stream) if rec is not None else ())

    def serve_connection(self, conn):
        """Answer one connection's requests until it closes (net.py:110-170)."""
        peer = "client"
        try:
            while True:
                h, arr = recv(conn, self.frames)
                rec = None
                try:
                    peer = self._command(conn, h, arr, peer)
                finally:
                    with self.lock:
                        rec = self.recon
                    self._release(arr, rec)
        except (EOFError, ConnectionError, OSError):
            self.log(f"[server] {peer} disconnected")
        except Exception as e:                       # report, then drop the connection
            self.log(f"[server] error from {peer}: {e!r}")
            try:
                send(conn, {"error": repr(e)})
            except Exception:
                pass
        finally:
            conn.close()

    def _command(self, conn, h, arr, peer):
        cmd = h.get("cmd")
        if cmd == "hello":
            peer = h.get("role", "client")
            self.log(f"[server] {peer} connected")
            send(conn, {"ok": True})
        elif cmd == "geometry":
            # a copy: the received buffer goes back to the pool after this command
            geom = geometry_from_message(h, np.array(arr.numpy() if isinstance(arr, torch.Tensor) else arr))
            rec = self._new_scan(geom)
            self.log(f"[server] new scan: {geom.n_angles} projections {geom.rows}x{geom.cols} "
                     f"({h['kind']} beam), backend={rec.backend}")
            send(conn, {"ok": True})
        elif cmd == "projections":
            rec, _ = self._current()
            block = arr if arr.dtype == torch.float32 else arr.to(torch.float32)
            send(conn, {"ok": True, "n": int(rec.add_projections(h["indices"], block))})
        elif cmd == "raw_projections":
            rec, _ = self._current()
            send(conn, {"ok": True, "n": int(rec.add_raw_projections(h["indices"], arr))})
        elif cmd == "flat_dark":
            rec, _ = self._current()
            a = arr.numpy() if isinstance(arr, torch.Tensor) else np.asarray(arr)
            if a.dtype == np.int16:
                a = a.view(np.uint16)
            rec.set_flat_dark(a[0], a[1], bin=int(h.get("bin", 1)), flip_rows=bool(h.get("flip_rows", False)),
                              mode=h.get("mode", "flexray"))
            send(conn, {"ok": True})
        elif cmd == "reset":
            rec, _ = self._current()
            rec.reset()
            send(conn, {"ok": True})
        elif cmd == "end":
            rec, _ = self._current()
            self.log(f"[server] adapter finished ({rec.n} projections)")
            send(conn, {"ok": True})
        elif cmd == "info":
            with self.lock:
                rec = self.recon
            send(conn, {"ready": rec is not None, **(rec.info() if rec is not None else {})})
        elif cmd == "slice":
            rec, srv = self._current()
            img = srv.submit(h["origin"], h["normal"], n=int(h["n"]), zoom=float(h.get("zoom", 1.0)),
                             center=h.get("center")).result()
            data, extra = encode_image(img, h.get("encoding"))
            send(conn, {"version": rec.version, **extra}, data)
        elif cmd == "slices":
            rec, srv = self._current()
            futs = [srv.submit(r["origin"], r["normal"], n=int(r["n"]), zoom=float(r.get("zoom", 1.0)),
                               center=r.get("center")) for r in h["requests"]]
            imgs = [f.result() for f in futs]
            flat = np.concatenate([i.ravel() for i in imgs]) if imgs else np.zeros(0, np.float32)
            data, extra = encode_image(flat, h.get("encoding"))
            send(conn, {"version": rec.version, "sizes": [int(i.shape[0]) for i in imgs], **extra}, data)
        elif cmd == "set_cor":
            rec, _ = self._current()
            rec.set_cor_shift(float(h["px"]))
            send(conn, {"ok": True})
        elif cmd == "auto_cor":
            rec, _ = self._current()
            best, _ = rec.estimate_cor(verbose=False)
            send(conn, {"best": best})
        elif cmd == "preview":
            _, srv = self._current()
            vol, origin, spacing = srv.submit_preview(int(h.get("maxdim", 64))).result()
            send(conn, {"origin": [float(o) for o in origin], "spacing": float(spacing)}, vol)
        else:
            send(conn, {"error": f"unknown command {cmd!r}"})
        return peer


# ------------------------------------------------------------------ clients
class _Conn:
    """One authenticated connection; calls are serialised (net.py:180-192)."""

    def __init__(self, address, role):
        self.conn = Client(tuple(address), authkey=authkey())
        self.lock = threading.Lock()
        self.call({"cmd": "hello", "role": role})

    def call(self, header, array=None):
        with self.lock:
            send(self.conn, header, array)
            h, arr = recv(self.conn)
        if "error" in h:
            raise RuntimeError(h["error"])
        return h, arr

    def close(self):
        self.conn.close()


class RemoteReconstructor:
    """Viewer-side proxy with the interface the viewers use locally (net.py:195-256).
    encoding="bf16" asks for BF16 slice replies (half the bytes; decoded to float)."""

    def __init__(self, address, wait=True, encoding="f32"):
        self.address = tuple(address)
        self.encoding = encoding
        self._c = _Conn(self.address, "viewer")
        self._preview_conn = None
        info = self.info()
        while wait and not info.get("ready"):
            print("[viewer] waiting for the server to receive a scan ...")
            time.sleep(1.0)
            info = self.info()
        self.box = np.asarray(info["box"], dtype=np.float64)
        self.kind = info["kind"]
        self.native_pixel = float(info["native_pixel"])
        self.backend = "remote:" + str(info.get("backend", "?"))
        self.n_total = info["n_total"]

    def info(self):
        return self._c.call({"cmd": "info"})[0]

    @property
    def n(self):
        return self.info()["n"]

    @property
    def cor_shift(self):
        return self.info()["cor_shift"]

    def plane_size(self, normal):
        return plane_size_for_box(self.box, normal)

    def inside_box(self, pts):
        return np.all(np.abs(pts) <= self.box, axis=-1)

    @staticmethod
    def _request(origin, normal, n, zoom, center):
        return {"origin": [float(v) for v in origin], "normal": [float(v) for v in normal], "n": int(n),
                "zoom": float(zoom), "center": None if center is None else [float(v) for v in center]}

    def reconstruct_plane(self, origin, normal, n=256, size=None, zoom=1.0, center=None):
        pts, _ = slice_points(self.box, origin, normal, n, size, zoom, center)
        h = {"cmd": "slice", **self._request(origin, normal, n, zoom, center)}
        if self.encoding != "f32":
            h["encoding"] = self.encoding
        hr, img = self._c.call(h)
        return decode_image(hr, img).astype(np.float64), pts

    def reconstruct_planes(self, requests):
        """Several slices in one round trip ("slices"): list of float images."""
        h = {"cmd": "slices", "requests": [self._request(r["origin"], r["normal"], r.get("n", 256),
                                                         r.get("zoom", 1.0), r.get("center"))
                                           for r in requests]}
        if self.encoding != "f32":
            h["encoding"] = self.encoding
        hr, flat = self._c.call(h)
        flat = decode_image(hr, flat)
        out, o = [], 0
        for n in hr["sizes"]:
            out.append(flat[o:o + n * n].reshape(n, n).astype(np.float64))
            o += n * n
        return out

    def preview_volume(self, maxdim=64):
        if self._preview_conn is None:                  # its own connection: no UI blocking
            self._preview_conn = _Conn(self.address, "viewer-preview")
        h, vol = self._preview_conn.call({"cmd": "preview", "maxdim": int(maxdim)})
        return vol, np.asarray(h["origin"]), float(h["spacing"])

    def set_cor_shift(self, px):
        self._c.call({"cmd": "set_cor", "px": float(px)})

    def estimate_cor(self, verbose=True):
        best = self._c.call({"cmd": "auto_cor"})[0]["best"]
        if verbose:
            print(f"[viewer] server COR search: best shift {best:+.2f} px")
        return best, None

    def warmup(self):
        pass

    def close(self):
        for c in (self._c, self._preview_conn):
            if c is not None:
                c.close()


class RemoteSink:
    """Adapter side: sends the geometry, then projections (net.py:259-270); each call
    blocks until the server has accepted the views."""

    def __init__(self, address, geom):
        self._c = _Conn(tuple(address), "adapter")
        self._c.call(*geometry_message(geom))

    def add_projections(self, indices, block):
        h, _ = self._c.call({"cmd": "projections", "indices": [int(i) for i in np.asarray(indices).ravel()]},
                            np.asarray(block, dtype=np.float32))
        return h.get("n")

    def set_flat_dark(self, flat, dark, bin=1, flip_rows=False, mode="flexray"):
        f, d = np.asarray(flat), np.asarray(dark)
        f = f[None] if f.ndim == 2 else f
        d = d[None] if d.ndim == 2 else d
        if f.shape != d.shape:
            raise ValueError("flat and dark stacks must have the same shape to travel together")
        self._c.call({"cmd": "flat_dark", "bin": int(bin), "flip_rows": bool(flip_rows), "mode": mode},
                     np.stack([f, d]).astype(np.uint16))

    def add_raw_projections(self, indices, raw):
        h, _ = self._c.call({"cmd": "raw_projections", "indices": [int(i) for i in np.asarray(indices).ravel()]},
                            np.asarray(raw, dtype=np.uint16))
        return h.get("n")

    def reset(self):
        """A new scan with the same geometry (the server forgets the received views)."""
        self._c.call({"cmd": "reset"})

    def end(self):
        self._c.call({"cmd": "end"})

    def close(self):
        self._c.close()
