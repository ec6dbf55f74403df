"""Reversible-car games: relative 5D table solve and its readers."""
