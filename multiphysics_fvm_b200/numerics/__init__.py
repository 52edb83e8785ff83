"""Space and time schemes (mirror of the reference's src/numerics package)."""
