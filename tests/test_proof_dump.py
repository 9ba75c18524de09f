"""ProverTranscript::finalize's proof dump (verifier/transcript/src/transcript.rs:258-282): with
BINIUS_DUMP_PROOF naming a file, finalize also writes the proof bytes there.  Host code only (the
transcript lives on the host)."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_finalize_dumps_proof_bytes(tmp_path):
    path = tmp_path / "proof.bin"
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import binius64_b200 as bg\n"
        "t = bg.ProverTranscript()\n"
        "t.message(bytes(range(100)))\n"
        "t.sample()\n"
        "t.message(b'abc')\n"
        "sys.stdout.write(t.finalize().hex())\n" % ROOT)
    env = dict(os.environ, BINIUS_DUMP_PROOF=str(path))
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                         check=True).stdout
    assert path.read_bytes() == bytes.fromhex(out)
    assert len(out) // 2 == 103


def test_no_dump_without_the_variable(tmp_path):
    env = {k: v for k, v in os.environ.items() if k != "BINIUS_DUMP_PROOF"}
    code = ("import sys; sys.path.insert(0, %r)\nimport binius64_b200 as bg\n"
            "t = bg.ProverTranscript(); t.message(b'x'); t.finalize()\n" % ROOT)
    subprocess.run([sys.executable, "-c", code], env=env, cwd=tmp_path, check=True)
    assert list(tmp_path.iterdir()) == []
