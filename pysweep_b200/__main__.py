"""`python -m pysweep_b200 ...`: the reference's pysweep command line."""
from .commandline import main

main()
