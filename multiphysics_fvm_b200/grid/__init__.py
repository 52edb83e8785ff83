"""Grid geometry and boundary conditions (mirror of the reference's src/grid)."""
