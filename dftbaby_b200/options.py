"""Options of DFTBaby's command-line programs, taken from the keyword parameters of the functions they call
(DFTB/optparse.py:1783-1935, OptionParserFuncWrapper).

* Every keyword parameter with a default becomes an option ``--name`` (``--name=value`` or ``--name value``);
  list-valued defaults and keyword-only parameters (programmatic arguments) are not options.
* Defaults come from the function, then from the ``[DFTBaby]`` section of ``dftbaby.cfg`` in the working
  directory, then from the command line.
* Values of options whose default is an int or a float are converted to that type; the others are read
  as text, then "None" / "none" becomes None and Python literals (numbers, lists, tuples, strings) are
  evaluated; anything else stays text.  DFTBaby evaluates such text with ``eval``; only literals are
  evaluated here.
* An option that none of the functions has is an error.
"""
import ast
import configparser
import inspect
import sys


def _convert(value):
    """optparse.OptionParserFuncWrapper.convert_types (optparse.py:1873-1896), with literals only."""
    if not isinstance(value, str):
        return value
    if value in ("None", "none"):
        return None
    try:
        return ast.literal_eval(value)
    except (ValueError, SyntaxError):
        return value


class OptionParserFuncWrapper:
    def __init__(self, funcs, usage, section_headers=("DFTBaby",), config_file="dftbaby.cfg"):
        if not isinstance(funcs, (list, tuple)):
            funcs = [funcs]
        config = configparser.ConfigParser()
        config.read(config_file)
        self.usage = usage
        self.options = {}          # name -> (type, default)
        self.func_parameters = {}  # function -> its option names
        for func in funcs:
            names = []
            for p in inspect.signature(func).parameters.values():
                if p.default is inspect.Parameter.empty or p.kind in (p.VAR_KEYWORD, p.VAR_POSITIONAL,
                                                                       p.KEYWORD_ONLY):
                    continue
                default = p.default
                if isinstance(default, list):
                    continue
                kind = int if type(default) is int else float if type(default) is float else str
                for section in section_headers:
                    if config.has_option(section, p.name):
                        default = config.get(section, p.name)
                        break
                if kind is not str and isinstance(default, str):
                    default = kind(default)
                self.options[p.name] = (kind, default)
                names.append(p.name)
            self.func_parameters[self._key(func)] = names

    @staticmethod
    def _key(func):
        return getattr(func, "__qualname__", func.__name__), getattr(func, "__module__", "")

    def format_help(self):
        lines = [self.usage]
        for name, (kind, default) in sorted(self.options.items()):
            lines.append("  --%s  (%s) [default: %s]" % (name, kind.__name__, default))
        return "\n".join(lines)

    def parse_args(self, f=None, argv=None):
        """(options, positional arguments); with f only the options that are keywords of f."""
        argv = sys.argv[1:] if argv is None else list(argv)
        values = {name: default for name, (_, default) in self.options.items()}
        args = []
        i = 0
        while i < len(argv):
            a = argv[i]
            if a in ("-h", "--help"):
                print(self.format_help())
                raise SystemExit(0)
            if a.startswith("--"):
                name, eq, val = a[2:].partition("=")
                if name not in self.options:
                    raise SystemExit("%s\nerror: no such option: --%s" % (self.usage, name))
                if not eq:
                    i += 1
                    if i == len(argv):
                        raise SystemExit("%s\nerror: --%s option requires an argument" % (self.usage, name))
                    val = argv[i]
                kind = self.options[name][0]
                try:
                    values[name] = kind(val) if kind is not str else val
                except ValueError:
                    raise SystemExit("%s\nerror: option --%s: invalid %s value: %r" % (self.usage, name,
                                                                                       kind.__name__, val))
            else:
                args.append(a)
            i += 1
        opts = {k: _convert(v) for k, v in values.items()}
        if f is not None:
            keep = self.func_parameters[self._key(f)]
            opts = {k: v for k, v in opts.items() if k in keep}
        return opts, args
