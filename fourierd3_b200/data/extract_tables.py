"""Extract the per-element D3 parameter tables into ``d3_tables.npz``.

The tables are the reference package's data files (``data/cnref.pt``,
``data/rcov.pt``, ``data/sqrtQz.pt``, ``data/en.pt``, ``data/rcov_cn.pt``),
loaded by ``src/fourierd3/utils.py:76-127``. They are physical parameters
(reference coordination numbers, covalent radii, sqrt(Q) ratios,
electronegativities), not code; the drop-in must use the identical values,
including their float32 storage precision, so they are copied bit for bit.

Run once, with the reference checkout's data directory as the argument::

    python fourierd3_b200/data/extract_tables.py <reference checkout>/data

``reference-c6.pt`` is absent from the reference checkout; it is not
extracted (see ``fourierd3_b200/tables.py`` for how the C6 table is obtained).
"""
import os
import sys

import numpy as np
import torch


def main(src_dir: str) -> None:
    out = {}
    for name in ("cnref", "rcov", "sqrtQz", "en", "rcov_cn"):
        t = torch.load(os.path.join(src_dir, name + ".pt"), weights_only=True)
        out[name] = t.numpy().copy()
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "d3_tables.npz")
    np.savez(dst, **out)
    for k, v in out.items():
        print(k, v.shape, v.dtype)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: extract_tables.py <reference checkout>/data")
    main(sys.argv[1])
