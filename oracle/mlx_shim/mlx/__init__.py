"""numpy-backed mlx stand-in used only to generate golden vectors."""
