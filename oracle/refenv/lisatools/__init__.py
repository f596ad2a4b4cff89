"""Stand-in for the external ``lisatools`` package: orbits and A/E/T PSD only,
re-exported from the bbhx_b200 host-side model so reference and product share them."""
