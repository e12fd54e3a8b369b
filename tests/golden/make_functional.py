"""Fixtures from the reference's own functional test (test/functional/).

Writes, under tests/golden/functional/:
  PiCoPiC.json  the test's configuration template rendered as its driver
                renders it (test.py:118-122: macro_amount = 2.1e5; the data
                root is a placeholder);
  step80.json   its known answers (true_data/<E|H|J>/<r|phi|z>/rec/0-32_0-128/4.dat):
                mean, standard deviation and variance of each probe's
                frame 4, i.e. of the state after 81 steps.

Usage: python tests/golden/make_functional.py [--ref /path/to/reference]
"""
import argparse
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
COMPONENTS = [f"{f}/{a}" for f in ("E", "H", "J") for a in ("r", "phi", "z")]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="the reference checkout")
    args = ap.parse_args()
    src = os.path.join(args.ref, "test", "functional")
    out = os.path.join(HERE, "functional")
    os.makedirs(out, exist_ok=True)
    with open(os.path.join(src, "picopic.json.tmpl")) as f:
        text = f.read()
    text = text.replace("{{ macro_amount }}", "2.1e5").replace("{{ result_path }}", "./data")
    json.loads(text)  # the rendered template must be plain JSON
    with open(os.path.join(out, "PiCoPiC.json"), "w") as f:
        f.write(text)
    answers = {}
    for comp in COMPONENTS:
        path = os.path.join(src, "true_data", comp, "rec", "0-32_0-128", "4.dat")
        with open(path) as f:
            mean, std, var = (float(x) for x in f.read().split())
        answers[comp] = {"mean": mean, "std": std, "var": var}
    doc = {"probe": "rec/0-32_0-128", "frame": 4, "steps": 81, "rtol": 0.15,
           "source": "test/functional/true_data/*/*/rec/0-32_0-128/4.dat", "components": answers}
    with open(os.path.join(out, "step80.json"), "w") as f:
        json.dump(doc, f, indent=1)
    print("wrote", out)


if __name__ == "__main__":
    main()
