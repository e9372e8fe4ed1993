"""The oracle: a CPU restatement of the reference LBVH path, used only as test infrastructure."""
