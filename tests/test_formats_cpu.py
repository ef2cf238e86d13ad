"""Input readers: FASTA, gzipped FASTA and UCSC 2bit load to the same packed
block (record order, names, soft-masking, N runs), as hspZ requires
(src/sequence.rs:460-522, whose fixture records and expected block are
reused here).  The 2bit files are written byte by byte from the published
format, in both byte orders and in both versions."""
import gzip
import struct

import pytest

from hspz_b200 import sequence as S

RECORDS = [("chrA", b"ACGTacgtNNAACG"), ("chrB", b"ttttGCttttN")]
EXPECTED_BUF = b"ACGTacgtNNAACG&ttttGCttttN&"


def runs(seq: bytes, pred):
    out, i = [], 0
    while i < len(seq):
        if pred(seq[i]):
            s = i
            while i < len(seq) and pred(seq[i]):
                i += 1
            out.append((s, i - s))
        else:
            i += 1
    return out


def two_bit_bytes(records, end="<", version=0):
    """A .2bit image: header, length-prefixed index, then per record the
    base count, N blocks (all starts, then all sizes), mask blocks, a
    reserved word and the bases two bits each (T C A G = 0 1 2 3, first base
    in the high bits)."""
    off_fmt = "Q" if version == 1 else "I"
    code = {ord("T"): 0, ord("C"): 1, ord("A"): 2, ord("G"): 3}
    bodies = []
    for _, seq in records:
        nb = runs(seq, lambda b: b in b"Nn")
        mb = runs(seq, lambda b: 97 <= b <= 122)
        body = struct.pack(end + "II", len(seq), len(nb))
        body += b"".join(struct.pack(end + "I", s) for s, _ in nb) + b"".join(struct.pack(end + "I", l) for _, l in nb)
        body += struct.pack(end + "I", len(mb))
        body += b"".join(struct.pack(end + "I", s) for s, _ in mb) + b"".join(struct.pack(end + "I", l) for _, l in mb)
        body += struct.pack(end + "I", 0)
        packed = bytearray()
        for i in range(0, len(seq), 4):
            byte = 0
            for j in range(4):
                c = seq[i + j] if i + j < len(seq) else ord("T")
                byte |= code.get(c & ~0x20, 0) << (6 - 2 * j)
            packed.append(byte)
        bodies.append(body + bytes(packed))
    head = struct.pack(end + "IIII", 0x1A412743, version, len(records), 0)
    index_len = sum(1 + len(n) + struct.calcsize(off_fmt) for n, _ in records)
    off = len(head) + index_len
    index = b""
    for (name, _), body in zip(records, bodies):
        index += bytes([len(name)]) + name.encode() + struct.pack(end + off_fmt, off)
        off += len(body)
    return head + index + b"".join(bodies)


def fasta_text(records) -> bytes:
    return b"".join(b">" + n.encode() + b"\n" + s + b"\n" for n, s in records)


@pytest.fixture
def files(tmp_path):
    fa = tmp_path / "x.fa"
    fa.write_bytes(fasta_text(RECORDS))
    gz = tmp_path / "x.fa.gz"
    gz.write_bytes(gzip.compress(fasta_text(RECORDS)))
    out = {"fa": fa, "gz": gz}
    for end, ver in (("<", 0), (">", 0), ("<", 1)):
        p = tmp_path / f"x{'le' if end == '<' else 'be'}{ver}.2bit"
        p.write_bytes(two_bit_bytes(RECORDS, end, ver))
        out[p.stem] = p
    return out


def test_three_formats_load_to_the_same_block(files):
    g = S.load_genome(files["fa"])
    assert g.format == S.FASTA
    assert bytes(g.buf) == EXPECTED_BUF
    assert g.block_len == len(EXPECTED_BUF) - 1
    for key, fmt in (("gz", S.FASTA_GZ), ("xle0", S.TWO_BIT), ("xbe0", S.TWO_BIT), ("xle1", S.TWO_BIT)):
        o = S.load_genome(files[key])
        assert o.format == fmt, key
        assert bytes(o.buf) == EXPECTED_BUF, key
        assert o.block_len == g.block_len
        assert [(c.name, c.start, c.len) for c in o.chrs] == [(c.name, c.start, c.len) for c in g.chrs]
        assert o.digest() == g.digest(), key


def test_format_comes_from_magic_bytes_not_the_name(tmp_path, files):
    fake = tmp_path / "really_gzip.fa"
    fake.write_bytes(files["gz"].read_bytes())
    assert S.detect_format(fake) == S.FASTA_GZ
    tb = tmp_path / "genome.bin"
    tb.write_bytes(files["xle0"].read_bytes())
    assert S.detect_format(tb) == S.TWO_BIT
    assert S.read_records(tb)[1] == RECORDS


def test_fasta_details(tmp_path):
    p = tmp_path / "y.fa"
    # text before the first header is ignored; names are the first token;
    # CRLF and interior whitespace vanish; a header without a name is ""
    p.write_bytes(b"junk\n>r1 description here\r\nAC GT\r\nac\tgt\n>\nNN\n>r3\n")
    assert S.read_fasta(p) == [("r1", b"ACGTacgt"), ("", b"NN"), ("r3", b"")]
    # concatenated gzip members read as one stream
    q = tmp_path / "y.fa.gz"
    q.write_bytes(gzip.compress(b">a\nAC\n") + gzip.compress(b"GT\n>b\nT\n"))
    assert S.read_fasta(q) == [("a", b"ACGT"), ("b", b"T")]


def test_block_size_guard_and_prefix(files):
    g = S.load_genome(files["fa"], prefix="ref.")
    assert [c.name for c in g.chrs] == ["ref.chrA", "ref.chrB"]
    with pytest.raises(ValueError):
        S.load_genome(files["fa"], seq_block_size=10)


def test_reverse_complement_of_a_loaded_block(files):
    g = S.load_genome(files["xle0"])
    rc, rc_chrs = g.reverse_complement()
    assert bytes(rc) == b"NaaaaGCaaaa&CGTTNNacgtACGT"
    assert [(c.name, c.start, c.len) for c in rc_chrs] == [("chrB", 0, 11), ("chrA", 12, 14)]
