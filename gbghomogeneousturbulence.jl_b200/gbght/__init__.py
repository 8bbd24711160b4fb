"""Host side of the B200 IF-RK time step (placeholder; the ctypes binding follows)."""
