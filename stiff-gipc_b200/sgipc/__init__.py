"""sgipc — B200-native per-Newton-iteration linear system of StiffGIPC (host side)."""
