"""Test infrastructure: CPU checkers (C restatement + reference build recipe). Never imported by the product."""
