"""Test-infrastructure oracle (CPU restatement of the reference). Never imported by
the product package ``fasteig_b200``."""
