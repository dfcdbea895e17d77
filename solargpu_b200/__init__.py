"""B200-native annual DSM irradiance path (viewshed DDA tracer, Perez solar
pass, CSR / ba-RLE reflection) behind the SolarGPU drop-in entry points."""
