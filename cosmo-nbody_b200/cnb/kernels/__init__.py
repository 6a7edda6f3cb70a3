"""Drop-in replacements for the reference's src/kernels modules."""
