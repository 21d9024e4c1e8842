"""CPU oracle (test infrastructure only): an FP64 C restatement of the MDFT
energy-and-gradient path of the reference.  Never imported by the product."""
