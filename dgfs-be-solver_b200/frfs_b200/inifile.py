# -*- coding: utf-8 -*-
"""Configuration reader with frfs's ``Inifile`` semantics.

Same behaviour as frfs/inifile.py:19-141 for the calls the DGFS hot path
makes: case-preserving keys, ``;`` inline comments, ``get(section, option,
default)`` that records the default when the option is absent, typed getters
and ``items_as``.
"""

import configparser
import os
import re

_sentinel = object()


class Inifile:
    def __init__(self, inistr=None):
        self._cp = cp = configparser.ConfigParser(
            inline_comment_prefixes=[';'], interpolation=None)
        cp.optionxform = str
        if inistr:
            cp.read_string(inistr)

    @staticmethod
    def load(file):
        if isinstance(file, str):
            with open(file) as fh:
                return Inifile(fh.read())
        return Inifile(file.read())

    def set(self, section, option, value):
        if not self._cp.has_section(section):
            self._cp.add_section(section)
        self._cp.set(section, option, str(value))

    def hasopt(self, section, option):
        return self._cp.has_option(section, option)

    def sections(self):
        return self._cp.sections()

    def get(self, section, option, default=_sentinel):
        if not self._cp.has_option(section, option):
            if default is _sentinel:
                raise configparser.NoOptionError(option, section)
            self.set(section, option, default)
        return os.path.expandvars(self._cp.get(section, option))

    def getpath(self, section, option, default=_sentinel, abs=False):
        path = os.path.expanduser(self.get(section, option, default))
        return os.path.abspath(path) if abs else path

    def getfloat(self, section, option, default=_sentinel):
        return float(self.get(section, option, default))

    def getint(self, section, option, default=_sentinel):
        return int(self.get(section, option, default))

    def getbool(self, section, option, default=_sentinel):
        v = self.get(section, option, default)
        return str(v).strip().lower() in ('1', 'true', 'yes', 'on')

    def items(self, section):
        if not self._cp.has_section(section):
            return {}
        return dict(self._cp.items(section))

    def items_as(self, section, type):
        iv = {}
        for k, v in self.items(section).items():
            try:
                iv[k] = type(v)
            except ValueError:
                pass
        return iv

    def getexpr(self, section, option, default=_sentinel):
        expr = self.get(section, option, default)
        if not re.match(r'[A-Za-z0-9 \t\n\r.,+\-*/%()<>]+$', expr):
            raise ValueError(f'Invalid characters in expression {expr!r}')
        return expr

    def tostr(self):
        import io
        buf = io.StringIO()
        self._cp.write(buf)
        return buf.getvalue()
