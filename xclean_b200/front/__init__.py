"""Frontend: Shi-Tomasi + cell NMS, ORB-256, 1-D ZNCC stereo with affine LK, Hamming matching (device)."""
