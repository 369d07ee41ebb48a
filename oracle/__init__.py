"""TEST INFRASTRUCTURE: the CPU oracle (restatement of bowshock's FP64 engine)."""
