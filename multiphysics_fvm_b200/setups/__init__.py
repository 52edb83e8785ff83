"""Setup files (reference schema, setups/*.py get_setup) for the benchmark
configurations: kelvin_helmholtz_sharp (2D KH, and its 3D extrusion),
rayleigh_taylor_3d, maxwell_spherical_pulse, heat_cylindrical_hotspot."""
