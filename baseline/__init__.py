"""Comparators that are not the product (the plain-GPU transliteration)."""
