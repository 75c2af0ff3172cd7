"""Train the cost model on a timing database and report its regret.

    python -m mex_linear_algebra_b200.train_costmodel --train train.json --eval eval.json \
        --out mex_linear_algebra_b200/costmodel.json

Training runs on the GPU in the library's own kernels.  The report compares,
on the evaluation records (every variant timed), the total time of the
model's choices with the exhaustive best (regret) and with the fixed rule.
"""
import argparse
import json

from . import costmodel


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", required=True)
    ap.add_argument("--eval", required=True)
    ap.add_argument("--out", default=costmodel.DEFAULT_MODEL)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--lr", type=float, default=3e-3)
    a = ap.parse_args()
    train = json.load(open(a.train))
    ev = json.load(open(a.eval))
    params, loss = costmodel.train(train, steps=a.steps, lr=a.lr)
    rep_train = costmodel.evaluate(params, train)
    rep_eval = costmodel.evaluate(params, ev)
    costmodel.save(params, a.out, meta={"train_records": len(train), "eval_records": len(ev),
                                        "final_loss": loss, "eval": rep_eval, "train": rep_train})
    print(json.dumps({"final_loss": loss, "train": rep_train, "eval": rep_eval}, indent=1))


if __name__ == "__main__":
    main()
