"""B200 lattice update for multiphaseLB (placeholder; filled in below)."""
