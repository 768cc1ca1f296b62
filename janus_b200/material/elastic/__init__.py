"""Elastic materials."""
