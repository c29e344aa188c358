"""Extract the reference's own known-answer vectors into reference_kats.json.

Reads lambda_vm's Rust test sources AS TEXT (nothing is compiled or run) and
records the pinned values those tests assert:
  * Keccak-256 vectors: crypto/ethrex-crypto/src/tests/keccak_tests.rs:57-79
  * transcript duplex KAT: crypto/crypto/src/tests/default_transcript_tests.rs:253-281
  * FRI query counts: crypto/stark/src/tests/proof_options_tests.rs:4-40
  * grinding nonces: crypto/stark/src/tests/grinding_tests.rs (seed, nonce,
    grinding factor, valid or not)
The JSON is committed so tests never need the reference tree at run time.
Usage: python tests/golden/extract_kats.py REFERENCE_ROOT
(REFERENCE_ROOT: the root of a lambda_vm checkout.)
"""
import json
import os
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/extract_kats.py REFERENCE_ROOT  (the root of a lambda_vm checkout)")
ROOT = sys.argv[1]
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")


def read(rel):
    with open(os.path.join(ROOT, rel)) as f:
        return f.read()


def keccak_kats():
    src = read("crypto/ethrex-crypto/src/tests/keccak_tests.rs")
    out = []
    for msg, hexd in re.findall(r'check_keccak_kat\(\s*b"([^"]*)",\s*"([0-9a-f]{64})"', src):
        out.append({"msg": msg, "digest": hexd})
    return out


def transcript_kat():
    src = read("crypto/crypto/src/tests/default_transcript_tests.rs")
    body = src[src.index("fn pinned_duplex_sample_semantics_across_refill"):]
    label = re.search(r'DefaultTranscript::<GoldilocksField>::new\(b"([^"]+)"\)', body).group(1)
    phase = re.search(r'te\.append_bytes\(b"([^"]+)"\)', body).group(1)
    u64_bound = re.search(r"t\.sample_u64\(1 << (\d+)\)", body).group(1)

    def arr(name):
        m = re.search(name + r": \[u64; \d+\] = \[([^\]]+)\]", src)
        return [int(x) for x in re.findall(r"\d+", m.group(1))]

    kat_u64 = int(re.search(r"const KAT_U64: u64 = (\d+);", src).group(1))
    return {"label": label, "base": arr("KAT_BASE"), "u64_bound_log2": int(u64_bound),
            "u64": kat_u64, "ext3_phase": phase, "ext3": arr("KAT_EXT3")}


def query_counts():
    src = read("crypto/stark/src/tests/proof_options_tests.rs")
    body = src[src.index("fn jbr_queries_match_expected_values"):]
    body = body[: body.index("\n}\n")]
    out = []
    for kind, args, q in re.findall(
            r"GoldilocksCubicProofOptions::(with_blowup|with_params)\(([^)]*)\)\s*\.unwrap\(\)\s*\.fri_number_of_queries,\s*(\d+)",
            body):
        a = [int(x) for x in args.split(",")]
        if kind == "with_blowup":
            a = [a[0], 128, 20]
        out.append({"blowup": a[0], "security_bits": a[1], "grinding": a[2], "queries": int(q)})
    return out


def grinding_kats():
    src = read("crypto/stark/src/tests/grinding_tests.rs")
    out = []
    for body in re.findall(r"#\[test\]\s*fn \w+\(\) \{(.*?)\n\}", src, re.S):
        seed = [int(x) for x in re.findall(r"\d+", re.search(r"let seed = \[([^\]]+)\]", body).group(1))]
        nonce = int(re.search(r"let nonce = (0x[0-9a-fA-F]+|\d+);", body).group(1), 0)
        g = int(re.search(r"let grinding_factor = (\d+);", body).group(1))
        valid = "assert!(!is_valid_nonce" not in body
        out.append({"seed": seed, "nonce": nonce, "grinding_factor": g, "valid": valid})
    return out


def main():
    kats = {
        "source": "lambda_vm test sources (text-extracted by tests/golden/extract_kats.py)",
        "keccak256": keccak_kats(),
        "transcript": transcript_kat(),
        "fri_queries": query_counts(),
        "grinding": grinding_kats(),
    }
    with open(OUT, "w") as f:
        json.dump(kats, f, indent=1)
    print(OUT)


if __name__ == "__main__":
    main()
