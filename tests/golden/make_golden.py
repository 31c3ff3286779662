"""Regenerates tests/golden/reference_fixtures.json from the reference tree.

Run in a checkout that has the rust-igraph sources, passing their path as
the first argument (or in $RUST_IGRAPH_REF); the GPU box never runs this.
It collects, unchanged:

* the conformance fixtures the reference's own tests replay for this path
  (tests/conformance/{c,py,r}/{pagerank,pagerank_weighted,personalized_pagerank}/*.json,
  driven by tests/conformance.rs:980-985, :3924-3970, :19492-19542) with the
  tolerance each driver applies;
* the generator fixtures (erdos_renyi_gnm, barabasi_game_bag, sbm_game) whose
  parameters and invariants (vcount, ecount, directedness) pin the seeded
  generators the benchmark inputs are built with;
* the golden 5-cycle personalized vector from the in-module test
  src/algorithms/properties/personalized_pagerank.rs:463-481 (parsed from
  the source text, tolerance 1e-6 as that test uses);
* the edge-list fixture fixtures/karate.edges that the reference's tests read
  with read_edgelist (tests/infomap.rs:11-15 and others), verbatim, with the
  vertex and edge counts its header states.
"""
import glob
import json
import os
import re
import sys

# the reference checkout: first argument, else $RUST_IGRAPH_REF
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RUST_IGRAPH_REF", "")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_fixtures.json")

# tolerance rules of the reference drivers
TOL = {
    "pagerank": {"kind": "rel", "tol": 1e-12, "driver": "tests/conformance.rs:44-67,980-985"},
    "pagerank_weighted": {"kind": "abs", "tol": 1e-6, "driver": "tests/conformance.rs:3924-3970"},
    "personalized_pagerank": {"kind": "rel", "tol": 1e-10, "driver": "tests/conformance.rs:19492-19542"},
}


def main():
    if not REF or not os.path.isdir(REF):
        sys.exit("usage: make_golden.py <path of the rust-igraph checkout> (or set RUST_IGRAPH_REF)")
    cases = []
    for algo in ("pagerank", "pagerank_weighted", "personalized_pagerank"):
        for path in sorted(glob.glob(os.path.join(REF, "tests/conformance/*", algo, "*.json"))):
            d = json.load(open(path))
            cases.append({
                "name": os.path.relpath(path, REF),
                "algo": d["algo"],
                "n": d["graph"]["n"],
                "directed": d["graph"]["directed"],
                "edges": d["graph"]["edges"],
                "weights": d["graph"]["weights"],
                "params": d["params"],
                "expected": d["expected"],
                **{"tol_" + k: v for k, v in TOL[algo].items()},
            })
    src = open(os.path.join(REF, "src/algorithms/properties/personalized_pagerank.rs")).read()
    m = re.search(r"fn oracle_5_cycle_biased\(\).*?let expected = \[(.*?)\];", src, re.S)
    if not m:
        sys.exit("could not find the 5-cycle golden vector")
    exp = [float(x.replace("_", "")) for x in re.findall(r"[0-9_.]+", m.group(1))]
    cases.append({
        "name": "src/algorithms/properties/personalized_pagerank.rs:463-481 (oracle_5_cycle_biased)",
        "algo": "personalized_pagerank",
        "n": 5,
        "directed": False,
        "edges": [[0, 1], [1, 2], [2, 3], [3, 4], [4, 0]],
        "weights": None,
        "params": {"reset": [0.5, 0.2, 0.1, 0.1, 0.1], "damping": 0.85},
        "expected": exp,
        "tol_kind": "abs",
        "tol_tol": 1e-6,
        "tol_driver": "personalized_pagerank.rs:480 close(&pr, &expected, 1e-6)",
    })
    gens = []
    for algo in ("erdos_renyi_gnm", "barabasi_game_bag", "sbm_game"):
        for path in sorted(glob.glob(os.path.join(REF, "tests/conformance/*", algo, "*.json"))):
            d = json.load(open(path))
            gens.append({"name": os.path.relpath(path, REF), "algo": d["algo"], "params": d["params"],
                         "expected": d["expected"]})
    karate = open(os.path.join(REF, "fixtures/karate.edges")).read()
    hm = re.search(r"(\d+) vertices.*?(\d+) edges", karate.splitlines()[0])
    edgelists = [{"name": "fixtures/karate.edges", "text": karate, "vcount": int(hm.group(1)),
                  "ecount": int(hm.group(2)), "used_by": "tests/infomap.rs:11-15, tests/label_propagation.rs"}]
    json.dump({"source": "rust-igraph v0.7.0 reference tree", "cases": cases, "generators": gens,
               "edgelists": edgelists}, open(OUT, "w"), indent=1)
    print(f"wrote {len(cases)} cases to {OUT}")


if __name__ == "__main__":
    main()
