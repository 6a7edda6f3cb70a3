"""Drop-in replacements for the reference's src/core modules."""
