"""B200-native evaluator for the spline EAM/MEAM fitting objective of Meamzilla."""
