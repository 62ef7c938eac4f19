"""prolix_b200: a B200-native implicit-solvent (OBC2 GBSA) MD step."""
