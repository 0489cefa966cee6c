"""Placeholder for ``jax.scipy`` (imported, unused, by the reference)."""
