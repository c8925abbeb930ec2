"""wind_b200: B200-native batched stiff-ODE integrators (SIE / RK2)."""
