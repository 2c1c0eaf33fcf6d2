"""Small utilities with the reference's semantics.

* :func:`set_params` — params-dict update that rejects unknown keys with
  ``KeyError`` (pymopt/utils/utilities.py:22-32).
* :func:`calTime` — elapsed-time print (pymopt/utils/utilities.py:9-16).
* :class:`ToJsonEncoder` — JSON encoder for NumPy scalars/arrays
  (pymopt/utils/utilities.py:34-43).
* :func:`_deprecate_positional_args` — FutureWarning for positional use of
  keyword-only arguments (pymopt/utils/validation.py:13-47).
"""
from __future__ import annotations

import json
import warnings
from functools import wraps
from inspect import Parameter, signature

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


def _deprecate_positional_args(f):
    sig = signature(f)
    kwonly_args, all_args = [], []
    for name, param in sig.parameters.items():
        if param.kind == Parameter.POSITIONAL_OR_KEYWORD:
            all_args.append(name)
        elif param.kind == Parameter.KEYWORD_ONLY:
            kwonly_args.append(name)

    @wraps(f)
    def inner_f(*args, **kwargs):
        extra = len(args) - len(all_args)
        if extra <= 0:
            return f(*args, **kwargs)
        args_msg = ["{}={}".format(name, arg)
                    for name, arg in zip(kwonly_args[:extra], args[-extra:])]
        warnings.warn("Pass {} as keyword args. From version 0.25 passing these as "
                      "positional arguments will result in an error".format(", ".join(args_msg)),
                      FutureWarning)
        kwargs.update(zip(sig.parameters, args))
        return f(**kwargs)
    return inner_f
