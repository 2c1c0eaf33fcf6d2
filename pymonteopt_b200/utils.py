"""Small utilities with the reference's semantics.

* :func:`set_params` — params-dict update that rejects unknown keys with
  ``KeyError`` (pymopt/utils/utilities.py:22-32).
* :func:`calTime` — elapsed-time print (pymopt/utils/utilities.py:9-16).
* :class:`ToJsonEncoder` — JSON encoder for NumPy scalars/arrays
  (pymopt/utils/utilities.py:34-43).
"""
from __future__ import annotations

import json

import numpy as np


def calTime(end, start):
    elapsed = end - start
    q, mod = divmod(elapsed, 60)
    if q < 60:
        print("Calculation time: %d minutes %0.3f seconds." % (q, mod))
    else:
        q2, mod2 = divmod(q, 60)
        print("Calculation time: %d h %0.3f minutes." % (q2, mod2))


def set_params(data: dict, keys, *initial_data, **kwargs) -> None:
    for dictionary in initial_data:
        for key in dictionary:
            if key not in keys:
                raise KeyError(key)
            data[key] = dictionary[key]
    for key in kwargs:
        if key not in keys:
            raise KeyError(key)
        data[key] = kwargs[key]


class ToJsonEncoder(json.JSONEncoder):
    def default(self, obj):
        if isinstance(obj, np.integer):
            return int(obj)
        if isinstance(obj, np.floating):
            return float(obj)
        if isinstance(obj, np.ndarray):
            return obj.tolist()
        return super().default(obj)
