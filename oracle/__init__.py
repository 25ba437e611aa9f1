"""Test-only checkers: the C restatement of the reference decrypt path
(cmd_oracle.c) and the reference's own CPU/ decoder built from its sources
(_ref/).  Never imported by the product."""
