"""`python -m floodca_b200 --grid DIR ...`: see floodca_b200.cli."""
import sys

from .cli import main

sys.exit(main())
