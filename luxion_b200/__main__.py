"""python -m luxion_b200 SCENE [-e ENVMAP] [-i N] [-o NAME] [-dmis] [-emis] [-lock]"""
import sys

from .cli import main

sys.exit(main())
