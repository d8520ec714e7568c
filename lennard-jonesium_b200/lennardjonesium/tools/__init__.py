"""Small helpers of the Python layer: dataclass <-> INI / dict conversion, linspace, divide.

Same behaviour as the reference's tools package
(src/python/lennardjonesium/tools/ini_parsable.py:27-90, dict_parsable.py:24-63,
linspace.py:24-35) and of more_itertools.divide, which the reference's sweep uses.
"""

import configparser
import dataclasses


def _sections(obj):
    return [f.name for f in dataclasses.fields(obj)]


def _keys(section_obj):
    return [f.name for f in dataclasses.fields(section_obj)]


class INIParsable:
    """Mixin for nested dataclasses (sections of scalar fields) read from / written to .ini files.

    Only fields the dataclass defines are read; a value takes the type of the field's current value.
    """

    @classmethod
    def from_file(cls, filename):
        obj = cls()
        obj.read(filename)
        return obj

    def read(self, filename):
        cp = configparser.ConfigParser()
        cp.read(filename)
        for sec in _sections(self):
            if sec not in cp:
                continue
            section_obj = getattr(self, sec)
            for key in _keys(section_obj):
                if key not in cp[sec]:
                    continue
                current = getattr(section_obj, key)
                if isinstance(current, bool):
                    value = cp.getboolean(sec, key)
                elif isinstance(current, int):
                    value = cp.getint(sec, key)
                elif isinstance(current, float):
                    value = cp.getfloat(sec, key)
                else:
                    value = cp[sec][key]
                setattr(section_obj, key, value)

    def write(self, filename):
        cp = configparser.ConfigParser()
        for sec in _sections(self):
            section_obj = getattr(self, sec)
            cp[sec] = {key: str(getattr(section_obj, key)) for key in _keys(section_obj)}
        with open(filename, "w") as fh:
            cp.write(fh)


class DictParsable:
    """Mixin for nested dataclasses converted to / from nested dictionaries."""

    @classmethod
    def from_dict(cls, d):
        obj = cls()
        for sec in _sections(obj):
            if sec in d:
                section_obj = getattr(obj, sec)
                for key in _keys(section_obj):
                    if key in d[sec]:
                        setattr(section_obj, key, d[sec][key])
        return obj

    def to_dict(self):
        return {sec: {key: getattr(getattr(self, sec), key) for key in _keys(getattr(self, sec))}
                for sec in _sections(self)}


def linspace(start, stop, points, endpoint=True):
    """`points` evenly spaced floats from start to stop (stop included when endpoint)."""
    span = stop - start
    steps = (points - 1) if endpoint else points
    return [start + (k / steps) * span for k in range(points)]


def divide(n, iterable):
    """Split into n consecutive parts of near-equal length (the first len % n parts one longer)."""
    items = list(iterable)
    q, r = divmod(len(items), n)
    parts, pos = [], 0
    for k in range(n):
        size = q + (1 if k < r else 0)
        parts.append(items[pos:pos + size])
        pos += size
    return parts
