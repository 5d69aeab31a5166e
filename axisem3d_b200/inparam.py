"""The reference's five input files (inparam.model/nr/source/output/advanced.yaml), read as
its InparamYAML does (SOLVER/src/shared/io/inparam/InparamYAML.hpp): values are reached by
':'-joined paths, '[i]' indexes a list, '{i}' names the key of the i-th single-key item of a
list (list_of_sources:{0} is the first source's name), and '[?]' is a list's length.

Only reading happens here; what each value means is applied by the preloop
(axisem3d_b200/preloop.py).
"""
from __future__ import annotations

import os

import yaml

FILES = ("model", "nr", "source", "output", "advanced")


class InparamError(RuntimeError):
    """A missing or invalid parameter; messages follow "InparamYAML::get || ..."."""


def _bool(v):
    if isinstance(v, bool):
        return v
    s = str(v).strip().lower()
    if s in ("true", "yes", "on", "1"):
        return True
    if s in ("false", "no", "off", "0"):
        return False
    raise ValueError(v)


class InparamYAML:
    """One YAML file, queried by path."""

    def __init__(self, path: str):
        self.path = path
        # every scalar stays a string, as in yaml-cpp; get() casts on request
        with open(path) as f:
            self.root = yaml.load(f, Loader=yaml.BaseLoader) or {}

    def _walk(self, key: str):
        node = self.root
        for part in key.split(":"):
            if part == "[?]":
                if not isinstance(node, list):
                    raise InparamError("InparamYAML::get || %s is not a list. || File: %s" % (key, self.path))
                return len(node)
            if part.startswith("[") and part.endswith("]"):
                i = int(part[1:-1])
                if not isinstance(node, list) or i >= len(node):
                    raise InparamError("InparamYAML::get || Index out of range: %s || File: %s" % (key, self.path))
                node = node[i]
            elif part.startswith("{") and part.endswith("}"):
                i = int(part[1:-1])
                if not isinstance(node, list) or i >= len(node) or not isinstance(node[i], dict):
                    raise InparamError("InparamYAML::get || Invalid key: %s || File: %s" % (key, self.path))
                return next(iter(node[i]))
            else:
                if not isinstance(node, dict) or part not in node:
                    raise InparamError("InparamYAML::get || Key not found: %s || File: %s" % (key, self.path))
                node = node[part]
        return node

    def contains(self, key: str) -> bool:
        try:
            self._walk(key)
            return True
        except InparamError:
            return False

    def get(self, key: str, kind=str):
        v = self._walk(key)
        try:
            if kind is bool:
                return _bool(v)
            if kind is str:
                return str(v)
            return kind(v)
        except (TypeError, ValueError):
            raise InparamError("InparamYAML::get || Error casting %s to %s: %r || File: %s"
                               % (key, kind.__name__, v, self.path))

    def get_bounded(self, key: str, lo=None, hi=None, kind=float):
        v = self.get(key, kind)
        if (lo is not None and v < lo) or (hi is not None and v > hi):
            raise InparamError("InparamYAML::getWithBounds || %s = %r out of range [%s, %s] || File: %s"
                               % (key, v, lo, hi, self.path))
        return v

    def get_options(self, key: str, options: dict):
        v = self.get(key, str)
        if v not in options:
            raise InparamError("InparamYAML::getWithLimits || %s = %s is not one of %s || File: %s"
                               % (key, v, sorted(options), self.path))
        return options[v]

    def get_vector(self, key: str, kind=str):
        v = self._walk(key)
        if v is None:
            return []
        if not isinstance(v, list):
            raise InparamError("InparamYAML::getVector || %s is not a list || File: %s" % (key, self.path))
        try:
            return [(_bool(x) if kind is bool else kind(x)) for x in v]
        except (TypeError, ValueError):
            raise InparamError("InparamYAML::getVector || Error casting %s || File: %s" % (key, self.path))


class Inparam:
    """The five files of one input directory (inparam::setup)."""

    def __init__(self, input_dir: str):
        self.input_dir = input_dir
        for name in FILES:
            p = os.path.join(input_dir, "inparam.%s.yaml" % name)
            if not os.path.exists(p):
                raise InparamError("inparam::setup || Missing input file: %s" % p)
            setattr(self, name, InparamYAML(p))

    def path(self, fname: str) -> str:
        """io::popInputDir: a file named in the inputs, relative to the input directory."""
        return fname if os.path.isabs(fname) else os.path.join(self.input_dir, fname)
