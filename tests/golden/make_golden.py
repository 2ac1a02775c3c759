"""Write tests/golden/reference_known_answers.json.

The reference (Rust) cannot be built or run in this environment, so its own
tests' known answers are restated here as data, each with the file:line of
the reference test it comes from (paths relative to the reference project's
`my-version/` directory). `tests/test_oracle_golden.py` pins the CPU oracle
to every entry. Re-run this script only when an entry is added.
"""
import json
import os

GOLDEN = {
    "centred_ranks_doubled": {
        "source": "src/metrics.rs:2172-2200",
        "cases": [
            {"v": [10.0, 20.0, 30.0], "want": [-2, 0, 2]},
            {"v": [5.0, 5.0, 5.0, 5.0], "want": [0, 0, 0, 0]},
            {"v": [1.0, 2.0, 2.0], "want": [-2, 1, 1]},
            {"v": ["-0.0", 0.0, 1.0, 1.0, 1.0, 2.0], "want": [-4, -4, 1, 1, 1, 5]},
        ],
    },
    "rank_score": {
        "source": "src/metrics.rs:2225-2249",
        "y": [1.0, 2.5, 3.0, 4.0, 9.0],
        "cases": [
            {"pred": [-5.0, 0.0, 7.0, 8.0, 100.0], "signed": False, "want": 0.0},
            {"pred": [5.0, 4.0, 3.0, 2.0, 1.0], "signed": False, "want": 0.0},
            {"pred": [5.0, 4.0, 3.0, 2.0, 1.0], "signed": True, "want": 2.0},
            {"pred": [3.0, 3.0, 3.0, 3.0, 3.0], "signed": False, "want": 1.0},
            {"pred": ["nan", 0.0, 7.0, 8.0, 100.0], "signed": False, "want": "inf"},
        ],
        "constant_target": {"y": [2.0, 2.0, 2.0, 2.0, 2.0], "pred": [1.0, 2.0, 3.0, 4.0, 5.0],
                            "want": 1.0},
        "one_row": {"y": [1.0], "pred": [4.0], "want": 1.0},
    },
    "recover_sin": {
        "source": "tests/recover.rs:154-165",
        "note": "y = sin(1.7 x) on 41 points of [-2, 2]; fit sin(c*x) from c = 1 with 25 iters",
        "grid": [-2.0, 2.0, 41], "iters": 25, "max_squared_error": 1e-20, "c": 1.7,
    },
    "implicit_circle": {
        "source": "src/implicit.rs:423-495",
        "note": "16 points of the unit circle; x^2 + y^2 - 1 has distance < 1e-12 on every "
                "point, 7 * f has bit-identical distances, constants 0 and 3 score +inf, and "
                "fitting x^2 + y^2 - 4 (20 iters) recovers the radius within 1e-6",
        "points": 16, "on_circle_tol": 1e-12, "radius_tol": 1e-6, "iters": 20,
    },
    "erf": {
        "source": "src/expr.rs:930-1041 (finite everywhere, erf(+-inf) = +-1, erf(-0) = +0); "
                  "values are the standard error function",
        "cases": [[0.0, 0.0, 1.0], [0.5, 0.5204998778130465, 0.4795001221869535],
                  [1.0, 0.8427007929497149, 0.15729920705028513],
                  [-2.0, -0.9953222650189527, 1.9953222650189528],
                  [3.0, 0.9999779095030014, 2.209049699858544e-05]],
        "tol": 1e-14,
    },
    "aic": {
        "source": "src/metrics.rs:1128-1154",
        "cases": [{"n": 10, "rss": 2.0, "k": 3,
                   "aic": 10 * __import__("math").log(0.2) + 6.0,
                   "bic": 10 * __import__("math").log(0.2) + 3 * __import__("math").log(10.0),
                   "aicc": 10 * __import__("math").log(0.2) + 6.0 + 2 * 3 * 4 / 6.0}],
    },
}


def main():
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                       "reference_known_answers.json")
    with open(out, "w") as f:
        json.dump(GOLDEN, f, indent=1, sort_keys=True)
    print(out)


if __name__ == "__main__":
    main()
