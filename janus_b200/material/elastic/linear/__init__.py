"""Linear elastic materials."""
