"""pyrowave-encode / pyrowave-decode: YUV4MPEG2 in, .pyrowave container, YUV4MPEG2 out.

The container and the command lines are the reference's (encode.cpp, decode.cpp,
yuv4mpeg.cpp). On CPU the tools' own sources are built against a test-only shim
that puts the CPU oracle behind the same C API (tests/cli_oracle_shim.cpp); on a
GPU the shipped binaries run against the CUDA library. Either way every packet
must equal the oracle's packetized frame and every decoded frame the oracle's
decode, bit for bit.
"""
import os
import struct
import subprocess

import numpy as np
import pytest

import oracle as O
from pyrowave_b200 import build as lib_build
from pyrowave_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _plane_shapes(w, h, c444):
    if c444:
        return [(h, w)] * 3
    return [(h, w), ((h + 1) // 2, (w + 1) // 2), ((h + 1) // 2, (w + 1) // 2)]


def write_y4m(path, frames, w, h, c444, tags="F30:1 Ip A1:1", chroma_tag=None):
    """8-bit planes, or uint16 planes written as little-endian 16-bit samples (tag C420p10 etc.)."""
    ctag = chroma_tag if chroma_tag is not None else ("C444" if c444 else "C420jpeg")
    with open(path, "wb") as f:
        f.write(f"YUV4MPEG2 W{w} H{h} {tags} {ctag}\n".encode())
        for planes in frames:
            f.write(b"FRAME\n")
            for p in planes:
                dt = "<u2" if np.asarray(p).dtype == np.uint16 else np.uint8
                f.write(np.ascontiguousarray(p, dt).tobytes())


def read_y4m(path, c444):
    data = open(path, "rb").read()
    nl = data.index(b"\n")
    header = data[:nl].decode()
    tags = {t[0]: t[1:] for t in header.split()[1:]}
    w, h = int(tags["W"]), int(tags["H"])
    wide = tags["C"].endswith("p16")
    shapes = _plane_shapes(w, h, c444)
    pos, frames = nl + 1, []
    while pos < len(data):
        assert data[pos:pos + 6] == b"FRAME\n"
        pos += 6
        planes = []
        for s in shapes:
            n = s[0] * s[1] * (2 if wide else 1)
            planes.append(np.frombuffer(data[pos:pos + n], "<u2" if wide else np.uint8).reshape(s).astype(
                np.uint16 if wide else np.uint8))
            pos += n
        frames.append(planes)
    return header, frames


def up_convert16(plane, depth):
    """yuv4mpeg.cpp:191-213: min(1, v / (2^depth - 1)) * 65535 + 0.5, in float."""
    f = plane.astype(np.float32) / np.float32((1 << depth) - 1)
    return (np.minimum(np.float32(1.0), f) * np.float32(65535.0) + np.float32(0.5)).astype(np.uint16)


def read_container(path):
    data = open(path, "rb").read()
    assert data[:8] == b"PYROWAVE"
    params = struct.unpack("<8i", data[8:40])
    pos, packets = 40, []
    while pos < len(data):
        (n,) = struct.unpack("<I", data[pos:pos + 4])
        packets.append(data[pos + 4:pos + 4 + n])
        pos += 4 + n
    assert pos == len(data)
    return params, packets


def write_container(path, params, packets):
    with open(path, "wb") as f:
        f.write(b"PYROWAVE" + struct.pack("<8i", *params))
        for p in packets:
            f.write(struct.pack("<I", len(p)) + bytes(p))


def oracle_expect(frames, w, h, c444, budget):
    """Packetized frames (one packet each) and their decodes, from the oracle
    (16-bit decodes for uint16 frames)."""
    enc = O.Oracle(w, h, c444)
    dec = O.Oracle(w, h, c444)
    parser = dec.parser()
    packets, decoded = [], []
    for planes in frames:
        enc.encode(planes, budget)
        stream, pk = enc.packetize(budget + 64, budget + 64)
        assert len(pk) == 1
        off, size = int(pk[0][0]), int(pk[0][1])
        packet = stream[off:off + size].tobytes()
        packets.append(packet)
        assert parser.push(packet) and parser.ready()
        offs, payload = parser.get()
        pyr = dec.dequant(offs, payload)
        decoded.append(dec.idwt16(pyr) if planes[0].dtype == np.uint16 else dec.idwt(pyr))
        parser.mark_decoded()
    return packets, decoded


@pytest.fixture(scope="module")
def shim_tools(tmp_path_factory):
    """The tools' sources linked against the oracle shim (CPU, test only)."""
    O.lib()  # builds oracle/liboracle.so if needed
    out = tmp_path_factory.mktemp("cli_shim")
    oracle_dir = os.path.join(ROOT, "oracle")
    tools = {}
    for tool in lib_build.CLI_TOOLS:
        exe = str(out / tool)
        cmd = ["g++", "-O1", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"), "-I", oracle_dir,
               "-I", lib_build.CLI] + lib_build.cli_sources(tool) + [
            os.path.join(ROOT, "tests", "cli_oracle_shim.cpp"), "-o", exe, "-L", oracle_dir, "-l:liboracle.so",
            f"-Wl,-rpath,{oracle_dir}"]
        subprocess.run(cmd, check=True, capture_output=True, text=True)
        tools[tool] = exe
    return tools


def _run(exe, *args):
    return subprocess.run([exe, *map(str, args)], capture_output=True, text=True, timeout=600)


def _round_trip(tools, tmp_path, w, h, c444, nframes, budget, seed, tags="F30:1 Ip A1:1"):
    frames = [synth.synth_frame(w, h, c444, seed + i) for i in range(nframes)]
    y4m, wave, out = tmp_path / "in.y4m", tmp_path / "out.pyrowave", tmp_path / "out.y4m"
    write_y4m(y4m, frames, w, h, c444, tags)
    r = _run(tools["pyrowave-encode"], y4m, wave, budget)
    assert r.returncode == 0, r.stderr
    params, packets = read_container(wave)
    exp_packets, exp_decoded = oracle_expect(frames, w, h, c444, budget)
    assert len(packets) == nframes
    for i, (got, exp) in enumerate(zip(packets, exp_packets)):
        assert len(got) <= budget
        assert got == exp, f"frame {i}: packet differs from the oracle's"
    r = _run(tools["pyrowave-decode"], wave, out)
    assert r.returncode == 0, r.stderr
    header, decoded = read_y4m(out, c444)
    assert len(decoded) == nframes
    for i in range(nframes):
        for p in range(3):
            assert np.array_equal(decoded[i][p], exp_decoded[i][p]), f"frame {i} plane {p}"
    return params, header


def test_round_trip_420_container_fields(shim_tools, tmp_path):
    params, header = _round_trip(shim_tools, tmp_path, 96, 64, False, 3, 6000, 20,
                                 tags="F30000:1001 Ip A1:1 XCOLORRANGE=FULL")
    # width, height, YUV420P, 4:2:0, full range, 30000/1001 fps, reserved
    assert params == (96, 64, 0, 0, 1, 30000, 1001, 0)
    assert header == "YUV4MPEG2 W96 H64 F30000:1001 Ip A1:1 XCOLORRANGE=FULL C420"


def test_round_trip_444_odd_size(shim_tools, tmp_path):
    params, header = _round_trip(shim_tools, tmp_path, 70, 50, True, 2, 9000, 30)
    assert params == (70, 50, 1, 1, 0, 30, 1, 0)
    assert header == "YUV4MPEG2 W70 H50 F30:1 Ip A1:1 XCOLORRANGE=LIMITED C444"


def _frames16(w, h, c444, n, seed, depth):
    """n frames of depth-bit samples (the synthetic 8-bit frame widened, seeded low bits)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        planes = synth.synth_frame(w, h, c444, seed + i)
        out.append([((p.astype(np.uint16) << (depth - 8)) |
                     rng.integers(0, 1 << (depth - 8), p.shape, dtype=np.uint16)) for p in planes])
    return out


def _round_trip16(tools, tmp_path, w, h, c444, nframes, budget, seed, depth):
    """A depth-bit stream: read and up-converted to 16 bits (the oracle codes
    the up-converted planes), written back as a 16-bit stream."""
    frames = _frames16(w, h, c444, nframes, seed, depth)
    tag = ("C444p" if c444 else "C420p") + str(depth)
    y4m, wave, out = tmp_path / "in16.y4m", tmp_path / "out16.pyrowave", tmp_path / "out16.y4m"
    write_y4m(y4m, frames, w, h, c444, chroma_tag=tag)
    r = _run(tools["pyrowave-encode"], y4m, wave, budget)
    assert r.returncode == 0, r.stderr
    params, packets = read_container(wave)
    up = [[up_convert16(p, depth) for p in f] for f in frames]
    exp_packets, exp_decoded = oracle_expect(up, w, h, c444, budget)
    assert packets == exp_packets
    r = _run(tools["pyrowave-decode"], wave, out)
    assert r.returncode == 0, r.stderr
    header, decoded = read_y4m(out, c444)
    assert header.endswith("C444p16" if c444 else "C420p16")
    for i in range(nframes):
        for p in range(3):
            assert decoded[i][p].dtype == np.uint16
            assert np.array_equal(decoded[i][p], exp_decoded[i][p]), f"frame {i} plane {p}"
    return params


def test_round_trip_16_bit(shim_tools, tmp_path):
    # 10-bit 4:2:0: the container records the 16-bit 4:2:0 format (2) the planes were coded from.
    params = _round_trip16(shim_tools, tmp_path, 96, 64, False, 2, 8000, 90, 10)
    assert params[:4] == (96, 64, 2, 0)
    # 16-bit 4:4:4 at an odd size.
    params = _round_trip16(shim_tools, tmp_path, 70, 50, True, 2, 12000, 95, 16)
    assert params[:4] == (70, 50, 3, 1)


def test_eight_frames_wrap_the_sequence_number(shim_tools, tmp_path):
    # The 3-bit sequence number wraps after 8 frames; each frame still decodes.
    _round_trip(shim_tools, tmp_path, 64, 64, False, 10, 3000, 40)


def test_decoder_assembles_frames_split_over_packets(shim_tools, tmp_path):
    w, h, budget = 128, 96, 12000
    frames = [synth.synth_frame(w, h, False, 50 + i) for i in range(2)]
    enc, ref = O.Oracle(w, h, False), O.Oracle(w, h, False)
    parser = ref.parser()
    packets, expect = [], []
    for planes in frames:
        enc.encode(planes, budget)
        stream, pk = enc.packetize(1024, budget + 64)
        assert len(pk) > 2
        for off, size in pk:
            packets.append(stream[int(off):int(off) + int(size)].tobytes())
            assert parser.push(packets[-1])
        assert parser.ready()
        offs, payload = parser.get()
        expect.append(ref.idwt(ref.dequant(offs, payload)))
        parser.mark_decoded()
    wave, out = tmp_path / "split.pyrowave", tmp_path / "split.y4m"
    write_container(wave, (w, h, 0, 0, 0, 60, 1, 0), packets)
    r = _run(shim_tools["pyrowave-decode"], wave, out)
    assert r.returncode == 0, r.stderr
    _, decoded = read_y4m(out, False)
    assert len(decoded) == 2
    for i in range(2):
        for p in range(3):
            assert np.array_equal(decoded[i][p], expect[i][p])


def test_usage_and_input_errors(shim_tools, tmp_path):
    enc, dec = shim_tools["pyrowave-encode"], shim_tools["pyrowave-decode"]
    r = _run(enc)
    assert r.returncode == 1 and "Usage: pyrowave-encode" in r.stderr
    r = _run(dec, "a")
    assert r.returncode == 1 and "Usage: pyrowave-decode" in r.stderr
    frame = synth.synth_frame(64, 64, False, 1)
    cases = {
        "C422": ("unsupported chroma format", dict(chroma_tag="C422")),
    }
    for name, (msg, kw) in cases.items():
        y = tmp_path / f"{name}.y4m"
        write_y4m(y, [], 64, 64, False, **kw)
        r = _run(enc, y, tmp_path / "x.pyrowave", 4000)
        assert r.returncode == 1 and msg in r.stderr, (name, r.stderr)
    y = tmp_path / "odd.y4m"
    write_y4m(y, [], 63, 64, False)
    r = _run(enc, y, tmp_path / "x.pyrowave", 4000)
    assert r.returncode == 1 and "even width and height" in r.stderr
    y = tmp_path / "budget.y4m"
    write_y4m(y, [frame], 64, 64, False)
    for bad in ("0", "abc", "5000000000"):
        r = _run(enc, y, tmp_path / "x.pyrowave", bad)
        assert r.returncode == 1 and "bytes_per_frame" in r.stderr
    # A stream that ends inside its second frame: the first is written, then an error.
    y = tmp_path / "short.y4m"
    write_y4m(y, [frame, frame], 64, 64, False)
    data = open(y, "rb").read()
    open(y, "wb").write(data[:-100])
    r = _run(enc, y, tmp_path / "short.pyrowave", 4000)
    assert r.returncode == 1 and "ends inside a frame" in r.stderr
    _, packets = read_container(tmp_path / "short.pyrowave")
    assert len(packets) == 1
    y = tmp_path / "notyuv.y4m"
    y.write_bytes(b"RIFF....")
    r = _run(enc, y, tmp_path / "x.pyrowave", 4000)
    assert r.returncode == 1 and "not a YUV4MPEG2 stream" in r.stderr


def test_container_errors(shim_tools, tmp_path):
    dec = shim_tools["pyrowave-decode"]
    bad = tmp_path / "bad.pyrowave"
    bad.write_bytes(b"PYROWAVX" + struct.pack("<8i", 64, 64, 0, 0, 0, 60, 1, 0))
    r = _run(dec, bad, tmp_path / "o.y4m")
    assert r.returncode == 1 and "bad magic" in r.stderr
    for params, msg in (((64, 64, 0, 1, 0, 60, 1, 0), "disagree"), ((0, 64, 0, 0, 0, 60, 1, 0), "frame size"),
                        ((64, 64, 2, 1, 0, 60, 1, 0), "disagree"), ((64, 64, 7, 0, 0, 60, 1, 0), "format")):
        write_container(bad, params, [])
        r = _run(dec, bad, tmp_path / "o.y4m")
        assert r.returncode == 1 and msg in r.stderr, (params, r.stderr)
    # A truncated last packet: complete frames are kept, then an error.
    w, h, budget = 64, 64, 3000
    frames = [synth.synth_frame(w, h, False, 60 + i) for i in range(2)]
    packets, expect = oracle_expect(frames, w, h, False, budget)
    write_container(bad, (w, h, 0, 0, 0, 60, 1, 0), packets)
    data = open(bad, "rb").read()
    open(bad, "wb").write(data[:-10])
    r = _run(dec, bad, tmp_path / "o.y4m")
    assert r.returncode == 1 and "truncated packet" in r.stderr
    _, decoded = read_y4m(tmp_path / "o.y4m", False)
    assert len(decoded) == 1 and all(np.array_equal(decoded[0][p], expect[0][p]) for p in range(3))
    # A malformed packet.
    write_container(bad, (w, h, 0, 0, 0, 60, 1, 0), [b"\x01\x02\x03"])
    r = _run(dec, bad, tmp_path / "o.y4m")
    assert r.returncode == 1 and "malformed packet" in r.stderr


@pytest.mark.gpu
def test_shipped_tools_round_trip_on_gpu(gpu, tmp_path):
    """The built binaries against the CUDA library: same packets and decodes as the oracle."""
    tools = {t: os.path.join(lib_build.BIN, t) for t in lib_build.CLI_TOOLS}
    for exe in tools.values():
        assert os.access(exe, os.X_OK), f"{exe} is not built (python -m pyrowave_b200.build)"
    _round_trip(tools, tmp_path, 256, 144, False, 3, 16000, 70)
    _round_trip(tools, tmp_path, 200, 128, True, 2, 30000, 80)
    _round_trip16(tools, tmp_path, 256, 144, False, 2, 20000, 85, 10)
    _round_trip16(tools, tmp_path, 200, 128, True, 2, 40000, 88, 16)
